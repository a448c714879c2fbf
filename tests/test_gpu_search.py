"""GPU RkNN search (plain form) against the reference: bit-identical answers on
the same index, through the C ABI."""
import numpy as np
import pytest

from conftest import golden_results, have_ref
from oracle import data, idx, port

import hrnn_b200 as H

pytestmark = pytest.mark.gpu


def test_search_matches_reference_golden(golden_idx, golden_search):
    h = H.HRNN.load(golden_idx, 32)
    Q = golden_search["Q"]
    for i, (m, kp, ef, th, k) in enumerate(golden_search["sweep"]):
        got = h.search_rknn_batch(Q, int(m), int(kp), int(ef), threshold=float(th), k=int(k))
        exp = golden_results(golden_search, i)
        bad = [q for q in range(len(Q)) if not np.array_equal(got[q], exp[q])]
        assert not bad, (i, bad[:5])


def test_search_single_query_api(golden_idx, golden_search):
    h = H.HRNN.load(golden_idx, 32)
    Q = golden_search["Q"]
    exp = golden_results(golden_search, 3)
    m, kp, ef, th, k = golden_search["sweep"][3]
    for q in range(5):
        assert h.searchRknn(Q[q], int(m), float(th), int(k), int(kp), int(ef)) == [int(x) for x in exp[q]]


def test_search_uneven_batch_matches_oracle(golden_idx):
    f = idx.read_idx(golden_idx)
    O = port.OracleIndex(f)
    h = H.HRNN.load(golden_idx, 32)
    rng = np.random.default_rng(4)
    Q = data.mixture(300, 32, 12, 1.0, 11, 99)
    m = rng.integers(1, 30, 300)
    kp = rng.integers(1, 30, 300)
    ef = rng.integers(1, 120, 300)
    got = h.search_rknn_batch(Q, m, kp, ef, threshold=1.0, k=7)
    exp = O.search_batch(Q, m, kp, ef, threshold=1.0, k=7)
    assert all(np.array_equal(a, b) for a, b in zip(got, exp))


def test_serve_mode_matches_reference_semantics(golden_idx, golden_search):
    h = H.HRNN.load(golden_idx, 32)
    h.compactForServing(12)
    f = idx.read_idx(golden_idx)
    O = port.OracleIndex(f, max_k_serve=12)
    Q = golden_search["Q"]
    got = h.search_rknn_batch(Q, 10, 24, 40, threshold=1.0, k=10)
    exp = O.search_batch(Q, 10, 24, 40, threshold=1.0, k=10)
    assert all(np.array_equal(a, b) for a, b in zip(got, exp))
    with pytest.raises(H.HrnnError):
        h.search_rknn_batch(Q[:2], 10, 24, 40, threshold=1.0, k=13)


def test_search_empty_and_errors(golden_idx):
    h = H.HRNN.load(golden_idx, 32)
    assert h.search_rknn_batch(np.zeros((0, 32), np.float32), 1, 1, 1) == []
    r = H.HRNN(32, 10, 8, 32, 100, 8)
    with pytest.raises(H.HrnnError) as e:
        r.search_rknn_batch(np.zeros((1, 32), np.float32), 1, 1, 1)
    assert str(e.value) == "searchRknn: RKNNG not built"


@pytest.mark.skipif(not have_ref(), reason="reference library oracle/_ref not built")
def test_search_matches_live_reference_d128(tmp_path):
    from oracle import ref
    X = data.mixture(20000, 128, 32, 1.0, 0, 0)
    Q = data.mixture(400, 128, 32, 1.0, 0, 1)
    r = ref.RefIndex.create(128, 20000, 16, 100, 100, 64)
    r.add_points(X, threads=16)
    r.refine(2, 20, threads=16)
    r.build_rknng()
    p = str(tmp_path / "r.idx")
    r.save(p)
    h = H.HRNN.load(p, 128)
    for m, kp, ef, th in ((1, 64, 50, 1.0), (5, 64, 100, 1.0), (10, 32, 200, 1.0), (20, 64, 64, 2.0),
                          (50, 64, 200, 1.0)):
        a = r.search_batch(Q, m, kp, ef, threshold=th, k=10)
        b = h.search_rknn_batch(Q, m, kp, ef, threshold=th, k=10)
        bad = [q for q in range(len(Q)) if not np.array_equal(a[q], b[q])]
        assert not bad, (m, kp, ef, th, bad[:5])
