"""Learned search budget: the device MLP against the FP64 oracle (forward and
gradients), training, and the learned search's answers against plain searches."""
import numpy as np
import pytest

from oracle import data, mlp

import hrnn_b200 as H

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def _model(seed=3):
    h = H.HRNN(32, 16, 8, 32, 100, 8)
    params = mlp.init_params(seed)
    h.budget_set_weights(params)
    return h, params


def test_budget_weights_roundtrip():
    h, params = _model()
    got = h.budget_get_weights()
    assert all(np.array_equal(a, b) for a, b in zip(got, params))


def test_budget_forward_matches_oracle():
    h, params = _model()
    X = np.random.default_rng(1).standard_normal((300, 256)).astype(np.float32)
    z = h.budget_predict(X)
    ref = mlp.forward(params, X, bf16_ops=True)[4]
    # BF16 operands as on the device, FP32 accumulation vs FP64.  An activation
    # within FP32 rounding of a BF16 rounding boundary can round the other way
    # (about 3e-5 of the 512 hidden activations of a row, so a few percent of the
    # rows): one BF16 ulp of one operand moves a logit by ~2^-8 |a| |w| < 2e-3.
    err = np.abs(z - ref)
    assert np.median(err) <= 1e-6
    assert np.mean(err > 1e-5) < 0.06
    assert np.max(err) <= 2e-3


@pytest.mark.parametrize("B", [1, 64, 333])
def test_budget_gradients_match_oracle(B):
    h, params = _model(5)
    rng = np.random.default_rng(B)
    X = rng.standard_normal((B, 256)).astype(np.float32)
    Y = rng.integers(0, 2, (B, 2)).astype(np.uint8)
    grads, loss = h.budget_gradients(X, Y)
    ref_loss, ref = mlp.loss_and_grads(params, X, Y, bf16_ops=True)
    assert abs(loss - ref_loss) <= 1e-5 * max(1.0, abs(ref_loss))
    for t, (g, r) in enumerate(zip(grads, ref)):
        # relative Frobenius error of each parameter's gradient; FP32 vs FP64 sums
        assert _rel(g, r) < 1e-3, (t, _rel(g, r))
    # and within BF16 rounding of the unrounded FP64 gradients
    _, exact = mlp.loss_and_grads(params, X, Y, bf16_ops=False)
    for t, (g, r) in enumerate(zip(grads, exact)):
        assert _rel(g, r) < 3e-2, (t, _rel(g, r))


def test_budget_training_learns_separable_task():
    h, _ = _model(9)
    rng = np.random.default_rng(2)
    X = rng.standard_normal((8192, 256)).astype(np.float32)
    Y = np.stack([X[:, 0] > 0, X[:, 0] + X[:, 1] > 0.5], 1).astype(np.uint8)
    _, l0 = h.budget_gradients(X[:2048], Y[:2048])
    loss = h.budget_train(X, Y, epochs=15, batch=256, lr=2e-3, seed=4)
    assert loss < 0.5 * l0
    Xt = rng.standard_normal((2048, 256)).astype(np.float32)
    Yt = np.stack([Xt[:, 0] > 0, Xt[:, 0] + Xt[:, 1] > 0.5], 1)
    acc = np.mean((h.budget_predict(Xt) > 0) == Yt)
    assert acc > 0.9, acc


def test_budget_errors():
    h = H.HRNN(32, 16, 8, 32, 100, 8)
    with pytest.raises(H.HrnnError):
        h.set_budget(True)  # no weights yet
    with pytest.raises(H.HrnnError):
        h.budget_predict(np.zeros((2, 256), np.float32))
    h.budget_set_weights(mlp.init_params(0))
    with pytest.raises(H.HrnnError):
        h.set_budget(True, m0=4, m1=2)
    with pytest.raises(H.HrnnError):
        h.set_budget(True, m0=1, m1=40)
    with pytest.raises(H.HrnnError):
        h.set_budget(True, confidence=0.3)


def _sets(res):
    return [frozenset(int(x) for x in r) for r in res]


@pytest.mark.parametrize("efl", [0, 40])
def test_learned_search_answers_equal_plain_searches(golden_idx, efl):
    """Every query's answer equals the plain search at the level the MLP chose
    (m_l proxies from the caller's beam, or from a beam of efl in two-pass mode)
    or at the caller's budget for the other queries."""
    h = H.HRNN.load(golden_idx, 32)
    m, kp, ef, k = 24, 24, 96, 10
    m0, m1, conf = 1, 3, 0.8
    ef_l = efl or ef
    Qtr = data.mixture(3000, 32, 12, 1.0, 11, 5)
    full = _sets(h.search_rknn_batch(Qtr, m, kp, ef, 1.0, k))
    lab = []
    for ml in (m0, m1):
        got = _sets(h.search_rknn_batch(Qtr, ml, kp, ef_l, 1.0, k))
        lab.append([f <= g for f, g in zip(full, got)])
    Y = np.array(lab, np.uint8).T
    h.budget_set_weights(mlp.init_params(1))
    h.set_budget(True, m0, m1, efl, conf)
    feat = h.budget_features(Qtr, k, m, ef)
    assert feat.shape == (3000, 256) and np.all(np.isfinite(feat))
    h.budget_train(feat, Y, epochs=30, batch=256, lr=2e-3, seed=1)

    Q = data.mixture(700, 32, 12, 1.0, 11, 77)
    z = h.budget_predict(h.budget_features(Q, k, m, ef))
    p = 1.0 / (1.0 + np.exp(-z.astype(np.float64)))
    lvl = np.where(p[:, 0] >= conf, 0, np.where(p[:, 1] >= conf, 1, 2))
    got = h.search_rknn_batch(Q, m, kp, ef, 1.0, k)
    st = h.last_search_stats()
    assert sum(st["n_budget"]) == len(Q)
    border = np.min(np.abs(p - conf), 1) < 1e-4
    if not border.any():
        assert st["n_budget"] == [int(np.sum(lvl == i)) for i in range(3)]
    h.set_budget(False)
    plain = {
        0: h.search_rknn_batch(Q, m0, kp, ef_l, 1.0, k),
        1: h.search_rknn_batch(Q, m1, kp, ef_l, 1.0, k),
        2: h.search_rknn_batch(Q, m, kp, ef, 1.0, k),
    }
    bad = [q for q in range(len(Q)) if not border[q] and not np.array_equal(got[q], plain[lvl[q]][q])]
    assert not bad, bad[:5]


@pytest.mark.parametrize("efl", [0, 48])
@pytest.mark.parametrize("level", [0, 1, 2])
def test_learned_search_forced_levels(golden_idx, level, efl):
    """Weights that pin every query to one level: the answers equal that level's
    plain search, and switching the budget off restores the caller's search."""
    h = H.HRNN.load(golden_idx, 32)
    m, kp, ef, k = 20, 24, 80, 9
    m0, m1 = 2, 5
    params = [np.zeros(s, np.float32) for s in H.BUDGET_SHAPES]
    params[5][:] = {0: (20, 20), 1: (-20, 20), 2: (-20, -20)}[level]
    h.budget_set_weights(params)
    h.set_budget(True, m0, m1, efl, 0.95)
    Q = data.mixture(400, 32, 12, 1.0, 11, 31)
    got = h.search_rknn_batch(Q, m, kp, ef, 1.0, k)
    st = h.last_search_stats()
    exp_counts = [0, 0, 0]
    exp_counts[level] = len(Q)
    assert st["n_budget"] == exp_counts
    h.set_budget(False)
    ef_l = efl or ef
    exp = h.search_rknn_batch(Q, (m0, m1, m)[level], kp, (ef_l, ef_l, ef)[level], 1.0, k)
    assert all(np.array_equal(a, b) for a, b in zip(got, exp))
    assert h.last_search_stats()["n_budget"] == [0, 0, 0]
