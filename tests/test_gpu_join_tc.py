"""Local join of refineKNNG on the tensor cores (BF16 Gram screen, exact FP32 for the
pairs it keeps) against the exact join: the same proposals and, state for state,
the same lists (up to the order of exactly equal distances), and in audit mode no
proposal that the screen would have dropped."""
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


def _same_up_to_ties(a, b, K):
    """Equal counts and bitwise-equal distances; ids equal except inside runs of
    exactly equal distances, which may hold them in another order (the device
    merge takes windows of one target's proposals in bucket order), and the run a
    full list cuts at K, which may keep another id of that distance."""
    (ai, ad, ac), (bi, bd, bc) = a, b
    assert np.array_equal(ac, bc)
    for i in range(len(ac)):
        c = int(ac[i])
        da, db = ad[i, :c].view(np.uint32), bd[i, :c].view(np.uint32)
        assert np.array_equal(da, db), i
        if np.array_equal(ai[i, :c], bi[i, :c]):
            continue
        s = 0
        while s < c:
            e = s + 1
            while e < c and da[e] == da[s]:
                e += 1
            if not np.array_equal(ai[i, s:e], bi[i, s:e]):
                assert e - s > 1, (i, s)
                assert np.array_equal(np.sort(ai[i, s:e]), np.sort(bi[i, s:e])) or e == c == K, (i, s)
            s = e


def _steps(p, d, mode, K, iters=3, sample=50):
    """One refineKNNG iteration at a time in `mode` and in the exact mode, both
    restarted from the exact run's lists after every step (each call starts with
    every entry new, hrnn.h:1742-1747), so the modes are compared state for state."""
    ht, he = H.HRNN.load(p, d), H.HRNN.load(p, d)
    ht.set_join_mode(mode)
    he.set_join_mode(H.JOIN_EXACT)
    stats = []
    for _ in range(iters):
        ht.refineKNNG(1, sample)
        he.refineKNNG(1, sample)
        st, se = ht.last_refine_stats(), he.last_refine_stats()
        assert st["join_mode"] == mode and se["join_mode"] == H.JOIN_EXACT
        assert st["join_dists"] == se["join_dists"]   # the reference's pair count
        assert st["proposals"] == se["proposals"]     # the same proposals
        ex = he.get_knng()
        _same_up_to_ties(ht.get_knng(), ex, K)
        ht.set_knng(*ex)
        stats.append(st)
    return stats


@pytest.mark.parametrize("d", [128, 96, 64])
def test_tensor_join_equals_exact_join(tmp_path, d):
    p = _pre_index(tmp_path, 20000, d, 100, 3)
    stats = _steps(p, d, H.JOIN_TENSOR, 100)
    # the screen leaves a minority of the pairs to exact FP32 once lists are full
    last = stats[-1]
    assert last["screen_survivors"][0] < 0.5 * last["join_dists"][0], last


@pytest.mark.parametrize("offset", [0.0, 40.0])
def test_audit_counts_no_screen_miss(tmp_path, offset):
    """offset 40 puts every point far from the origin: the Gram form cancels
    badly, the error term grows with the norms, most pairs stay for exact FP32
    (the dense pass) and the decisions must still be safe."""
    p = _pre_index(tmp_path, 30000, 128, 100, 4, offset)
    stats = _steps(p, 128, H.JOIN_AUDIT, 100)
    assert sum(s["screen_misses"][0] for s in stats) == 0, [s["screen_misses"] for s in stats]
    assert sum(s["screen_survivors"][0] for s in stats) > 0


def test_join_mode_argument_checked(tmp_path):
    p = _pre_index(tmp_path, 2000, 32, 20, 5)
    h = H.HRNN.load(p, 32)
    with pytest.raises(H.HrnnError):
        h.set_join_mode(7)


def test_tensor_join_falls_back_beyond_one_tile(tmp_path):
    """S = 80 gives sample lists of up to 160 new rows, more than one M = 128 tile:
    the refinement runs the exact join (and says so) with the same lists."""
    p = _pre_index(tmp_path, 6000, 64, 60, 6)
    ht, he = H.HRNN.load(p, 64), H.HRNN.load(p, 64)
    ht.set_join_mode(H.JOIN_TENSOR)
    ht.refineKNNG(1, 80)
    he.refineKNNG(1, 80)
    assert ht.last_refine_stats()["join_mode"] == H.JOIN_EXACT
    _same_up_to_ties(ht.get_knng(), he.get_knng(), 60)
