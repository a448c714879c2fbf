"""The float64 RkNN ground-truth generator (hrnn_b200.groundtruth) on the GPU
against an exact float64 numpy brute force of the definition of
scripts/gen_rknn_gt.py:5-8 (RkNN(q) = { x : ||q - x||^2 <= ||x - x_k||^2 }),
including exact boundary cases (duplicated points, queries equal to points: a
distance of 0 against a k-th radius of 0), and through its command line in the
file layout of scripts/gen_rknn_gt.py:10-14."""
import numpy as np
import pytest

from oracle import data

pytestmark = pytest.mark.gpu


def _points():
    X = data.mixture(30000, 96, 40, 1.0, 21, 21)
    # 30 points repeated 12 times: their k-th radius (k = 10) is exactly 0
    dup = X[:30]
    X = np.concatenate([X, np.repeat(dup, 11, axis=0)])
    Q = data.mixture(300, 96, 40, 1.0, 21, 22)
    Q[:5] = dup[:5]                       # at distance 0 from a point of radius 0
    Q[5:10] = X[1000:1005]                # equal to ordinary points
    return X, Q


def test_groundtruth_gpu_matches_float64_brute_force(tmp_path):
    import torch
    from hrnn_b200 import groundtruth as G
    X, Q = _points()
    k = 10
    dev = torch.device("cuda", 0)
    kth = G.kth_radius_fp64(X, k, dev, chunk=2048)
    ref_kth = data.kth_nn_fp64(X, k)
    assert np.all(kth[:30] == 0.0) and np.all(ref_kth[:30] == 0.0)
    assert np.allclose(kth, ref_kth, rtol=1e-12, atol=0)
    gt = G.rknn_fp64(X, Q, kth, dev, chunk=64)
    ref = data.rknn_gt_fp64(X, Q, ref_kth)
    bad = [i for i, ((ids, _), r) in enumerate(zip(gt, ref)) if not np.array_equal(np.sort(ids), r)]
    assert not bad, f"queries {bad[:8]} differ from the brute force"
    for j in range(5):                    # the duplicated point and its 11 copies answer it
        assert {0 + j} | {30000 + 11 * j + t for t in range(11)} <= set(gt[j][0].tolist())
    for ids, ds in gt:
        assert np.all(np.diff(ds) >= 0)


def test_groundtruth_cli_file_layout(tmp_path):
    from hrnn_b200 import groundtruth as G
    X, Q = _points()
    Q = Q[:64]
    pb, pq, po = str(tmp_path / "base.fbin"), str(tmp_path / "query.fbin"), str(tmp_path / "gt.bin")
    G.write_fbin(pb, X)
    G.write_fbin(pq, Q)
    assert G.main(["--base", pb, "--query", pq, "--k", "10", "--output", po, "--chunk_base", "1024",
                   "--chunk_query", "32"]) == 0
    raw = open(po, "rb").read()
    nq = int(np.frombuffer(raw, np.uint32, 1, 0)[0])
    off = np.frombuffer(raw, np.uint32, nq + 1, 4)
    tot = int(off[-1])
    ids = np.frombuffer(raw, np.uint32, tot, 4 + 4 * (nq + 1))
    ds = np.frombuffer(raw, np.float32, tot, 4 + 4 * (nq + 1) + 4 * tot)
    assert nq == len(Q) and len(raw) == 4 + 4 * (nq + 1) + 8 * tot
    ref_kth = data.kth_nn_fp64(X, 10)
    ref = data.rknn_gt_fp64(X, Q, ref_kth)
    Xd, Qd = X.astype(np.float64), Q.astype(np.float64)
    for i in range(nq):
        s = slice(int(off[i]), int(off[i + 1]))
        assert np.array_equal(np.sort(ids[s]), ref[i])
        exp_d = ((Xd[ids[s]] - Qd[i]) ** 2).sum(1).astype(np.float32)
        assert np.allclose(ds[s], exp_d, rtol=1e-6, atol=0)  # ids ordered by distance, distances stored
        assert np.all(np.diff(ds[s]) >= 0)
