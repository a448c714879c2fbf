"""What the trained budget network gains over the method without it, on queries
it never saw.  An MLP trained by the library's own kernels on (query, "is the
answer with m_l proxies complete") labels of a training stream serves a
held-out stream: against the plain search at the caller's m it must scan far
fewer postings per query (the work of phase B/C) at the same recall, and
against a plain search whose uniform m costs at least as many postings it must
reach at least that search's recall -- the budget spends the work where a query
needs it."""
import numpy as np
import pytest

from oracle import data

import hrnn_b200 as H

pytestmark = pytest.mark.gpu

N, D, K, KP, EF, KK = 30000, 64, 64, 64, 96, 10
M_USER, M0, M1 = 12, 1, 3


@pytest.fixture(scope="module")
def setup():
    X = data.mixture(N, D, 48, 1.0, 41, 41)
    h = H.HRNN(D, N, 16, 100, 100, K)
    h.add_points(X)
    h.refineKNNG(4, 20)
    h.buildRKNNG()
    Qtr = data.mixture(8000, D, 48, 1.0, 41, 42)
    Qho = data.mixture(1500, D, 48, 1.0, 41, 43)
    kth = data.kth_nn_fp64(X, KK)
    gt = data.rknn_gt_fp64(X, Qho, kth)
    return X, h, Qtr, Qho, gt


def _sets(res):
    return [frozenset(int(x) for x in r) for r in res]


def _run(h, Q, m):
    res = h.search_rknn_batch(Q, m, KP, EF, 1.0, KK)
    st = h.last_search_stats()
    return res, st["n_posting"] / len(Q)


def test_trained_budget_cuts_work_at_equal_recall(setup):
    X, h, Qtr, Qho, gt = setup
    full = _sets(h.search_rknn_batch(Qtr, M_USER, KP, EF, 1.0, KK))
    Y = np.array([[f <= g for f, g in zip(full, _sets(h.search_rknn_batch(Qtr, ml, KP, EF, 1.0, KK)))]
                  for ml in (M0, M1)], np.uint8).T
    h.set_budget(False, M0, M1, 0, 0.9)
    feat = h.budget_features(Qtr, KK, M_USER, EF)
    h.budget_train(feat, Y, epochs=30, batch=256, lr=2e-3, seed=3)

    plain, post_plain = _run(h, Qho, M_USER)
    h.set_budget(True, M0, M1, 0, 0.9)
    try:
        learned, post_learned = _run(h, Qho, M_USER)
        levels = h.last_search_stats()["n_budget"]
    finally:
        h.set_budget(False)
    r_plain, r_learned = data.macro_recall(gt, plain), data.macro_recall(gt, learned)
    print(f"held-out: plain m={M_USER} recall {r_plain:.4f} postings/q {post_plain:.0f}; "
          f"learned recall {r_learned:.4f} postings/q {post_learned:.0f}, levels {levels}")
    assert levels[0] + levels[1] > 0.3 * len(Qho)         # the network takes the cheap levels often
    assert post_learned < 0.7 * post_plain                 # and cuts the scanned postings
    assert r_learned >= r_plain - 0.01                     # at the caller's recall

    # a uniform m with at least the learned form's postings: the learned form is
    # at least as accurate
    for m in range(1, M_USER + 1):
        res, post = _run(h, Qho, m)
        if post >= post_learned:
            r_m = data.macro_recall(gt, res)
            print(f"uniform m={m}: recall {r_m:.4f} postings/q {post:.0f}")
            assert r_learned >= r_m - 0.002, (m, r_m, r_learned)
            break
