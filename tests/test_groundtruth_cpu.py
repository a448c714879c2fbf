"""The float64 RkNN ground-truth generator (hrnn_b200.groundtruth) against the
numpy restatement of the definition (scripts/gen_rknn_gt.py:5-8), run on the
CPU device, and its file layout against the oracle's writer."""
import numpy as np
import pytest

from oracle import data


def test_groundtruth_matches_definition(tmp_path):
    torch = pytest.importorskip("torch")
    from hrnn_b200 import groundtruth as G
    X = data.mixture(700, 24, 6, 1.0, 5, 5)
    Q = data.mixture(60, 24, 6, 1.0, 5, 6)
    cpu = torch.device("cpu")
    kth = G.kth_radius_fp64(X, 7, cpu, chunk=128)
    ref_kth = data.kth_nn_fp64(X, 7)
    # float64 sums in different orders: equal to ~1e-15 relative
    assert np.allclose(kth, ref_kth, rtol=1e-12, atol=0)
    gt = G.rknn_fp64(X, Q, kth, cpu, chunk=16)
    ref = data.rknn_gt_fp64(X, Q, ref_kth)
    assert all(np.array_equal(np.sort(ids), r) for (ids, _), r in zip(gt, ref))
    for ids, ds in gt:
        assert np.all(np.diff(ds) >= 0)
    p1, p2 = str(tmp_path / "a.bin"), str(tmp_path / "b.bin")
    G.write_rknn_gt(p1, gt)
    data.write_rknn_gt(p2, X, Q, ref)
    back = G.read_rknn_gt(p1)
    assert all(np.array_equal(a[0], b[0]) for a, b in zip(back, gt))
    # same layout and ids as the oracle's writer (distances agree to float32)
    b1, b2 = open(p1, "rb").read(), open(p2, "rb").read()
    assert len(b1) == len(b2)
    nq = len(Q)
    tot = int(np.frombuffer(b1, np.uint32, 1, 4 + 4 * nq)[0])
    head = 4 + 4 * (nq + 1) + 4 * tot
    assert b1[:head] == b2[:head]


def test_fbin_roundtrip(tmp_path):
    from hrnn_b200 import groundtruth as G
    X = data.mixture(50, 8, 3, 1.0, 1, 1)
    p = str(tmp_path / "x.fbin")
    G.write_fbin(p, X)
    assert np.array_equal(G.read_fbin(p), X)
    assert np.array_equal(data.read_fbin(p), X)


def test_bounded_groundtruth_equals_full():
    """Radii only for the points an upper bound of their k-th radius lets some
    query reach: the same ground truth as with every radius, fewer radii."""
    torch = pytest.importorskip("torch")
    from hrnn_b200 import groundtruth as G
    X = data.mixture(3000, 24, 6, 1.0, 5, 5)
    Q = data.mixture(50, 24, 6, 1.0, 5, 6)
    cpu = torch.device("cpu")
    kth = G.kth_radius_fp64(X, 7, cpu, chunk=256)
    rows = np.array([5, 17, 2999])
    assert np.array_equal(G.kth_radius_fp64(X, 7, cpu, chunk=100, rows=rows), kth[rows])
    full = G.rknn_fp64(X, Q, kth, cpu, chunk=16)
    got, nr = G.rknn_fp64_bounded(X, Q, kth * 1.3 + 0.1, 7, cpu, q_chunk=16, x_chunk=1000)
    assert nr < len(X)
    assert all(np.array_equal(a[0], b[0]) for a, b in zip(full, got))
