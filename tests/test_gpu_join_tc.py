"""Local join of refineKNNG on the tensor cores (BF16 Gram screen, exact FP32 for the
pairs it keeps) against the exact join: the same lists bit for bit, and in audit
mode no proposal that the screen would have dropped."""
import numpy as np
import pytest

from oracle import data

import hrnn_b200 as H

pytestmark = pytest.mark.gpu


def _pre_index(tmp_path, n, d, K, seed, offset=0.0):
    X = data.mixture(n, d, 32, 1.0, seed, seed) + np.float32(offset)
    h = H.HRNN(dim=d, max_elements=n, M=16, ef_construction=100, random_seed=100, K_knng=K)
    h.add_points(np.ascontiguousarray(X, dtype=np.float32))
    p = str(tmp_path / f"pre_{d}_{seed}.idx")
    h.saveIndex(p)
    return p


def _refine(p, d, mode, iters, sample):
    h = H.HRNN.load(p, d)
    h.set_join_mode(mode)
    h.refineKNNG(iters, sample)
    return h.get_knng(), h.last_refine_stats()


def _assert_same(a, b):
    (ai, ad, ac), (bi, bd, bc) = a, b
    assert np.array_equal(ac, bc)
    for i in range(len(ac)):
        c = int(ac[i])
        assert np.array_equal(ai[i, :c], bi[i, :c]), i
        assert np.array_equal(ad[i, :c].view(np.uint32), bd[i, :c].view(np.uint32)), i


@pytest.mark.parametrize("d", [128, 96, 64])
def test_tensor_join_lists_equal_exact_join(tmp_path, d):
    p = _pre_index(tmp_path, 20000, d, 100, 3)
    exact, se = _refine(p, d, H.JOIN_EXACT, 4, 50)
    tens, st = _refine(p, d, H.JOIN_TENSOR, 4, 50)
    _assert_same(tens, exact)
    assert se["join_mode"] == H.JOIN_EXACT and st["join_mode"] == H.JOIN_TENSOR
    assert st["join_dists"] == se["join_dists"]        # the reference's pair count
    assert st["proposals"] == se["proposals"]
    # the screen leaves a minority of the pairs to exact FP32 once lists are full
    assert st["screen_survivors"][-1] < 0.5 * st["join_dists"][-1], st


@pytest.mark.parametrize("offset", [0.0, 40.0])
def test_audit_counts_no_screen_miss(tmp_path, offset):
    """offset 40 puts every point far from the origin: the Gram form cancels
    badly, the error term grows with the norms, most pairs stay for exact FP32
    (the dense pass) and the decisions must still be safe."""
    p = _pre_index(tmp_path, 30000, 128, 100, 4, offset)
    aud, sa = _refine(p, 128, H.JOIN_AUDIT, 4, 50)
    assert sa["join_mode"] == H.JOIN_AUDIT
    assert sum(sa["screen_misses"]) == 0, sa["screen_misses"]
    assert sum(sa["screen_survivors"]) > 0
    exact, _ = _refine(p, 128, H.JOIN_EXACT, 4, 50)
    _assert_same(aud, exact)


def test_join_mode_argument_checked(tmp_path):
    p = _pre_index(tmp_path, 2000, 32, 20, 5)
    h = H.HRNN.load(p, 32)
    with pytest.raises(H.HrnnError):
        h.set_join_mode(7)
