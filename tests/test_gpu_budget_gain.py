"""What the trained budget network gains over the method without it, on queries
it never saw.  An MLP trained by the library's own kernels on (query, "is the
answer with m_l proxies complete") labels of a training stream serves a
held-out stream.  Against the plain search's recall-versus-work curve (uniform
m = 1 .. the caller's m, postings scanned per query being the work of phase
B/C, linearly interpolated between neighbouring m), the budget must reach at
least the recall the plain search reaches with the same work -- it spends the
work where a query needs it -- and scan fewer postings than the caller's m."""
import numpy as np
import pytest

from oracle import data

import hrnn_b200 as H

pytestmark = pytest.mark.gpu

N, D, K, KP, EF, KK = 40000, 64, 64, 64, 96, 10
M_USER, M0, M1 = 5, 1, 3


@pytest.fixture(scope="module")
def setup():
    X = data.mixture(N, D, 48, 1.0, 41, 41)
    h = H.HRNN(D, N, 16, 100, 100, K)
    h.add_points(X)
    h.refineKNNG(4, 20)
    h.buildRKNNG()
    Qtr = data.mixture(30000, D, 48, 1.0, 41, 42)
    Qho = data.mixture(2000, D, 48, 1.0, 41, 43)
    kth = data.kth_nn_fp64(X, KK)
    gt = data.rknn_gt_fp64(X, Qho, kth)
    return X, h, Qtr, Qho, gt


def _sets(res):
    return [frozenset(int(x) for x in r) for r in res]


def _run(h, Q, m):
    res = h.search_rknn_batch(Q, m, KP, EF, 1.0, KK)
    st = h.last_search_stats()
    return res, st["n_posting"] / len(Q)


def test_trained_budget_spends_work_where_it_pays(setup):
    X, h, Qtr, Qho, gt = setup
    full = _sets(h.search_rknn_batch(Qtr, M_USER, KP, EF, 1.0, KK))
    Y = np.array([[f <= g for f, g in zip(full, _sets(h.search_rknn_batch(Qtr, ml, KP, EF, 1.0, KK)))]
                  for ml in (M0, M1)], np.uint8).T
    h.set_budget(False, M0, M1, 0, 0.9)
    feat = h.budget_features(Qtr, KK, M_USER, EF)
    h.budget_train(feat, Y, epochs=30, batch=256, lr=2e-3, seed=3)

    plain, post_plain = _run(h, Qho, M_USER)
    r_plain = data.macro_recall(gt, plain)
    uniform = []
    for m in range(1, M_USER + 1):
        res, post = _run(h, Qho, m)
        uniform.append((m, post, data.macro_recall(gt, res)))
    print(f"held-out: plain m={M_USER} recall {r_plain:.4f} postings/q {post_plain:.0f}")
    posts = np.array([u[1] for u in uniform])
    recs = np.array([u[2] for u in uniform])
    for conf in (0.99, 0.998):
        h.set_budget(True, M0, M1, 0, conf)
        try:
            learned, post_learned = _run(h, Qho, M_USER)
            levels = h.last_search_stats()["n_budget"]
        finally:
            h.set_budget(False)
        r_learned = data.macro_recall(gt, learned)
        r_eq = float(np.interp(post_learned, posts, recs))  # the plain curve at the same work
        print(f"confidence {conf}: learned recall {r_learned:.4f} postings/q {post_learned:.0f} levels {levels}; "
              f"plain at equal work {r_eq:.4f}; uniform {[(m, round(p_), round(r_, 4)) for m, p_, r_ in uniform]}")
        assert levels[0] + levels[1] > 0.1 * len(Qho)      # the network takes the cheap levels
        assert post_learned < post_plain                    # less work than the caller's m
        assert r_learned >= r_eq - 0.002                     # at least the plain search's recall for that work
