"""The reduced-precision search path: the two-parent beam search (beam_fast.cuh)
and the streaming INT8 verification (k_verify_stream).

* On the same proxies the streaming verification answers exactly as the CTA
  table kernel (HRNN_VERIFY=table forces the latter), overflow pass included.
* Every point the INT8 form returns passes the reference's exact test (FP32 L2 in
  the reference's order against the stored k-th distance), up to the FP64
  re-decisions inside the tie band, and its recall stays at the exact form's.
* The learned budget's two-pass mode stores the frontier beam and a fallback
  query resumes it: with the level beam as large as the caller's the resumed
  search has nothing left to do and answers exactly as a fresh search; with a
  smaller level beam its answers keep exact decisions and the fresh search's
  recall."""
import os

import numpy as np
import pytest

from oracle import data, idx, port

import hrnn_b200 as H

pytestmark = pytest.mark.gpu


def _build(dim, n=20000, K=64, seed=31):
    X = data.mixture(n, dim, 32, 1.0, seed, seed)
    Q = data.mixture(400, dim, 32, 1.0, seed, seed + 1)
    h = H.HRNN(dim, n, 16, 100, 100, K)
    h.add_points(X)
    h.refineKNNG(4, 20)
    h.buildRKNNG()
    return X, Q, h


@pytest.fixture(scope="module")
def idx128():
    return _build(128)


@pytest.fixture(scope="module")
def idx96():
    return _build(96, seed=33)


def _with_table(h, Q, m, kp, ef, k, th=1.0):
    os.environ["HRNN_VERIFY"] = "table"
    try:
        return h.search_rknn_batch(Q, m, kp, ef, threshold=th, k=k)
    finally:
        del os.environ["HRNN_VERIFY"]


@pytest.mark.parametrize("which", ["idx128", "idx96"])
def test_stream_verification_equals_table(request, which):
    X, Q, h = request.getfixturevalue(which)
    h.set_precision(H.PREC_INT8)
    try:
        for m, kp, ef, k in ((5, 64, 100, 10), (1, 64, 40, 10), (12, 32, 64, 5), (40, 64, 100, 64)):
            a = h.search_rknn_batch(Q, m, kp, ef, threshold=1.0, k=k)
            sa = h.last_search_stats()
            b = _with_table(h, Q, m, kp, ef, k)
            bad = [i for i in range(len(Q)) if not np.array_equal(a[i], b[i])]
            assert not bad, (m, kp, ef, k, bad[:5])
            assert sa["n_result"] == sum(len(x) for x in a)
        # the last case has answers of hundreds of points: some queries took the
        # overflow pass of the streaming kernel
        assert max(len(x) for x in a) > 100
    finally:
        h.set_precision(H.PREC_FP32_EXACT)


def _exact_fails(X, Q, h, res, k):
    ids, d, cnt = h.get_knng()
    bad = 0
    for qi, r in enumerate(res):
        for lab in r:
            i = int(lab)  # labels are the insertion order here
            d32 = port.l2(Q[qi], X[i])
            kd = d[i, k - 1] if cnt[i] > k - 1 else np.float32(np.finfo(np.float32).max)
            bad += not (d32 <= kd)
    return bad


@pytest.mark.parametrize("which", ["idx128", "idx96"])
def test_int8_form_exact_decisions_and_recall(request, which):
    X, Q, h = request.getfixturevalue(which)
    kth = data.kth_nn_fp64(X, 10)
    gt = data.rknn_gt_fp64(X, Q, kth)
    plain = h.search_rknn_batch(Q, 5, 64, 100, k=10)
    h.set_precision(H.PREC_INT8)
    try:
        fast = h.search_rknn_batch(Q, 5, 64, 100, k=10)
        st = h.last_search_stats()
    finally:
        h.set_precision(H.PREC_FP32_EXACT)
    assert _exact_fails(X, Q, h, fast, 10) <= st["n_fp64_flipped"]
    assert data.macro_recall(gt, fast) >= data.macro_recall(gt, plain) - 0.01
    assert st["n_expanded"] > 0 and st["n_dist"] > st["n_expanded"]


def _forced_budget(h, level, m0, m1, efl):
    params = [np.zeros(s, np.float32) for s in H.BUDGET_SHAPES]
    params[5][:] = {0: (20, 20), 1: (-20, 20), 2: (-20, -20)}[level]
    h.budget_set_weights(params)
    h.set_budget(True, m0, m1, efl, 0.95)


def test_resumed_fallback_equals_fresh_search_when_nothing_is_left(idx128):
    X, Q, h = idx128
    m, kp, ef, k = 6, 64, 96, 10
    h.set_precision(H.PREC_INT8)
    try:
        fresh = h.search_rknn_batch(Q, m, kp, ef, threshold=1.0, k=k)
        _forced_budget(h, 2, 1, 3, ef)      # level beam = the caller's: the stored beam is complete
        got = h.search_rknn_batch(Q, m, kp, ef, threshold=1.0, k=k)
        assert h.last_search_stats()["n_budget"] == [0, 0, len(Q)]
    finally:
        h.set_budget(False)
        h.set_precision(H.PREC_FP32_EXACT)
    assert all(np.array_equal(a, b) for a, b in zip(got, fresh))


@pytest.mark.parametrize("level", [0, 1, 2])
def test_two_pass_levels_with_resume(idx128, level):
    X, Q, h = idx128
    m, kp, ef, k, efl, m0, m1 = 6, 64, 128, 10, 32, 1, 3
    kth = data.kth_nn_fp64(X, k)
    gt = data.rknn_gt_fp64(X, Q, kth)
    h.set_precision(H.PREC_INT8)
    try:
        fresh = h.search_rknn_batch(Q, m, kp, ef, threshold=1.0, k=k)
        lvl = h.search_rknn_batch(Q, (m0, m1)[min(level, 1)], kp, efl, threshold=1.0, k=k)
        _forced_budget(h, level, m0, m1, efl)
        got = h.search_rknn_batch(Q, m, kp, ef, threshold=1.0, k=k)
        st = h.last_search_stats()
    finally:
        h.set_budget(False)
        h.set_precision(H.PREC_FP32_EXACT)
    exp = [0, 0, 0]
    exp[level] = len(Q)
    assert st["n_budget"] == exp
    if level < 2:   # levels take the first m_l entries of the level beam
        assert all(np.array_equal(a, b) for a, b in zip(got, lvl))
    else:           # resumed from the level beam: exact decisions, the fresh search's recall
        assert _exact_fails(X, Q, h, got, k) <= st["n_fp64_flipped"]
        assert data.macro_recall(gt, got) >= data.macro_recall(gt, fresh) - 0.01


def test_overlapped_second_search_equals_serial(idx128, monkeypatch):
    """Two-pass mode with a mix of levels: the fallback queries' second search runs
    on a second stream beside the verification of the others (two verification
    groups); the answers equal those of the serial order (HRNN_LEARNED_SERIAL=1)."""
    from oracle import mlp as OM
    X, Q, h = idx128
    m, kp, ef, k, efl = 6, 64, 128, 10, 32
    params = list(OM.init_params(5))[:6] + [np.zeros(H.BUDGET_IN, np.float32), np.ones(H.BUDGET_IN, np.float32)]
    params[5][:] = 0.0  # logits around 0: about half the queries pass a cutoff just above 0.5
    h.set_precision(H.PREC_INT8)
    try:
        h.budget_set_weights(params)
        h.set_budget(True, 1, 3, efl, 0.5001)
        over = h.search_rknn_batch(Q, m, kp, ef, threshold=1.0, k=k)
        lv = h.last_search_stats()["n_budget"]
        monkeypatch.setenv("HRNN_LEARNED_SERIAL", "1")
        serial = h.search_rknn_batch(Q, m, kp, ef, threshold=1.0, k=k)
        assert h.last_search_stats()["n_budget"] == lv
    finally:
        h.set_budget(False)
        h.set_precision(H.PREC_FP32_EXACT)
    assert 0 < lv[2] < len(Q) and lv[0] + lv[1] > 0, lv
    assert all(np.array_equal(a, b) for a, b in zip(over, serial))
