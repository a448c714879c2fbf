"""Captured search plans (hrnn_search_plan_*): the batch search recorded once as a
CUDA graph over fixed device buffers and replayed per batch.  Every replay must
answer exactly as the stream-ordered batch call does on the same inputs."""
import numpy as np
import pytest

from oracle import data

import hrnn_b200 as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def index(tmp_path_factory):
    X = data.mixture(20000, 128, 32, 1.0, 7, 7)
    h = H.HRNN(dim=128, max_elements=20000, M=16, ef_construction=100, random_seed=100, K_knng=100)
    h.add_points(X)
    h.refineKNNG(4, 30)
    h.buildRKNNG()
    return h


def _batch(seed, nq, m_max, ef_max):
    rng = np.random.default_rng(seed)
    Q = data.mixture(nq, 128, 32, 1.0, 7, 100 + seed)
    m = rng.integers(1, m_max + 1, nq).astype(np.uint32)
    ef = rng.integers(10, ef_max + 1, nq).astype(np.uint32)
    kp = rng.integers(20, 101, nq).astype(np.uint32)
    return Q, m, kp, ef


def _regular(h, torch, q, m, kp, ef, k, cap):
    off = torch.zeros(q.shape[0] + 1, dtype=torch.int64, device="cuda")
    lab = torch.zeros(cap, dtype=torch.int64, device="cuda")
    tot = h.search_rknn_batch_device(q.data_ptr(), q.shape[0], m.data_ptr(), kp.data_ptr(), ef.data_ptr(), 1.0, k,
                                     off.data_ptr(), lab.data_ptr(), cap)
    torch.cuda.synchronize()
    return off.cpu().numpy(), lab.cpu().numpy()[:tot]


@pytest.mark.parametrize("precision", [H.PREC_FP32_EXACT, H.PREC_INT8])
def test_plan_replays_equal_batch_calls(index, precision):
    import torch
    h = index
    h.set_precision(precision)
    nq, m_max, ef_max, k, cap = 3000, 8, 120, 10, 3000 * 64
    q = torch.zeros((nq, 128), dtype=torch.float32, device="cuda")
    m = torch.zeros(nq, dtype=torch.int32, device="cuda")
    kp = torch.zeros(nq, dtype=torch.int32, device="cuda")
    ef = torch.zeros(nq, dtype=torch.int32, device="cuda")
    off = torch.zeros(nq + 1, dtype=torch.int64, device="cuda")
    lab = torch.zeros(cap, dtype=torch.int64, device="cuda")
    plan = h.search_plan(q.data_ptr(), nq, m.data_ptr(), kp.data_ptr(), ef.data_ptr(), m_max, ef_max, 1.0, k,
                         off.data_ptr(), lab.data_ptr(), cap)
    try:
        for seed in (1, 2):  # two different batches through the same graph
            Q, hm, hkp, hef = _batch(seed, nq, m_max, ef_max)
            q.copy_(torch.from_numpy(Q))
            m.copy_(torch.from_numpy(hm.astype(np.int32)))
            kp.copy_(torch.from_numpy(hkp.astype(np.int32)))
            ef.copy_(torch.from_numpy(hef.astype(np.int32)))
            torch.cuda.synchronize()  # the plan runs on the index's stream
            plan.run()
            total, clamped = plan.result()
            assert not clamped
            got_off, got_lab = off.cpu().numpy(), lab.cpu().numpy()[:total]
            exp_off, exp_lab = _regular(h, torch, q, m, kp, ef, k, cap)
            assert total == exp_off[-1] and total > 0
            assert np.array_equal(got_off, exp_off)
            assert np.array_equal(got_lab, exp_lab)
        # the host-buffer run: the same batch copied in from host memory
        hq = np.ascontiguousarray(Q, np.float32)
        hm32, hkp32, hef32 = (np.ascontiguousarray(x, np.uint32) for x in (hm, hkp, hef))
        hoff = np.zeros(nq + 1, np.uint64)
        hlab = np.zeros(cap, np.uint64)
        total, clamped = plan.run_host(hq.ctypes.data, hm32.ctypes.data, hkp32.ctypes.data, hef32.ctypes.data,
                                       hoff.ctypes.data, hlab.ctypes.data, cap)
        assert not clamped and total == exp_off[-1]
        assert np.array_equal(hoff.astype(np.int64), exp_off)
        assert np.array_equal(hlab[:total].astype(np.int64), exp_lab)
    finally:
        plan.close()
        h.set_precision(H.PREC_FP32_EXACT)


@pytest.mark.parametrize("efl", [0, 48])
@pytest.mark.parametrize("precision", [H.PREC_INT8, H.PREC_BF16])
def test_plan_learned_budget_replays_equal_batch_calls(index, precision, efl):
    """The learned budget recorded in a plan (frontier pass, features, MLP, levels;
    in two-pass mode the second search, beside the first group's verification in
    the INT8 form): replays of two batches answer as the batch calls with the
    budget on, and a later change of the budget invalidates the plan."""
    import torch
    from oracle import mlp
    h = index
    h.set_precision(precision)
    nq, m_max, ef_max, k, cap = 3000, 8, 120, 10, 3000 * 64
    # labels a linear function of one input feature decides, so the model's
    # levels spread over the queries: level 0 above the median, level 1 above
    # the lower quartile, the caller's m below it
    Qtr = data.mixture(3000, 128, 32, 1.0, 7, 55)
    h.budget_set_weights(mlp.init_params(3))
    feat = h.budget_features(Qtr, k, 6, 100)
    f0 = feat[:, 0]
    Y = np.stack([f0 > np.median(f0), f0 > np.quantile(f0, 0.25)], 1).astype(np.uint8)
    h.budget_train(feat, Y, epochs=30, batch=256, lr=2e-3, seed=2)
    h.set_budget(True, 2, 4, efl, 0.8)
    q = torch.zeros((nq, 128), dtype=torch.float32, device="cuda")
    m = torch.zeros(nq, dtype=torch.int32, device="cuda")
    kp = torch.zeros(nq, dtype=torch.int32, device="cuda")
    ef = torch.zeros(nq, dtype=torch.int32, device="cuda")
    off = torch.zeros(nq + 1, dtype=torch.int64, device="cuda")
    lab = torch.zeros(cap, dtype=torch.int64, device="cuda")
    plan = h.search_plan(q.data_ptr(), nq, m.data_ptr(), kp.data_ptr(), ef.data_ptr(), m_max, ef_max, 1.0, k,
                         off.data_ptr(), lab.data_ptr(), cap)
    try:
        for seed in (1, 2):
            Q, hm, hkp, hef = _batch(seed, nq, m_max, ef_max)
            q.copy_(torch.from_numpy(Q))
            m.copy_(torch.from_numpy(hm.astype(np.int32)))
            kp.copy_(torch.from_numpy(hkp.astype(np.int32)))
            ef.copy_(torch.from_numpy(hef.astype(np.int32)))
            torch.cuda.synchronize()
            plan.run()
            total, clamped = plan.result()
            assert not clamped
            got_off, got_lab = off.cpu().numpy(), lab.cpu().numpy()[:total]
            exp_off, exp_lab = _regular(h, torch, q, m, kp, ef, k, cap)
            levels = h.last_search_stats()["n_budget"]
            assert sum(levels) == nq and levels[2] > 0 and levels[0] + levels[1] > 0, levels
            assert total == exp_off[-1] and total > 0
            assert np.array_equal(got_off, exp_off)
            assert np.array_equal(got_lab, exp_lab)
        h.set_budget(True, 2, 4, efl, 0.9)  # other settings: the plan records the old ones
        with pytest.raises(H.HrnnError) as e:
            plan.run()
        assert e.value.code == H.ERR_STATE
    finally:
        plan.close()
        h.set_budget(False)
        h.set_precision(H.PREC_FP32_EXACT)


@pytest.mark.parametrize("precision", [H.PREC_FP32_EXACT, H.PREC_INT8])
def test_plan_bounded_result_slices(index, precision, monkeypatch):
    """A plan whose per-query result slices are smaller than the queries' posting
    counts (the bounded staging of large indexes, forced small here): queries whose
    acceptances pass their slice go to the overflow pass, and the answers still
    equal the batch calls'."""
    import torch
    h = index
    h.set_precision(precision)
    nq, m_max, ef_max, k, cap = 2000, 8, 120, 10, 2000 * 64
    Q, hm, hkp, hef = _batch(5, nq, m_max, ef_max)
    q = torch.from_numpy(Q).cuda()
    m = torch.from_numpy(hm.astype(np.int32)).cuda()
    kp = torch.from_numpy(hkp.astype(np.int32)).cuda()
    ef = torch.from_numpy(hef.astype(np.int32)).cuda()
    exp_off, exp_lab = _regular(h, torch, q, m, kp, ef, k, cap)
    st = h.last_search_stats()
    # slices just long enough for the longest answer, shorter than most queries'
    # postings: acceptances (an owner counted once per proxy listing it) pass them
    slice_len = int(np.diff(exp_off).max()) + 8
    assert st["n_posting"] / nq > slice_len
    monkeypatch.setenv("HRNN_PLAN_MAX_SLICE", str(slice_len))
    off = torch.zeros(nq + 1, dtype=torch.int64, device="cuda")
    lab = torch.zeros(cap, dtype=torch.int64, device="cuda")
    plan = h.search_plan(q.data_ptr(), nq, m.data_ptr(), kp.data_ptr(), ef.data_ptr(), m_max, ef_max, 1.0, k,
                         off.data_ptr(), lab.data_ptr(), cap)
    try:
        torch.cuda.synchronize()
        plan.run()
        total, clamped = plan.result()
        assert not clamped
        got_off, got_lab = off.cpu().numpy(), lab.cpu().numpy()[:total]
        assert np.array_equal(got_off, exp_off)
        assert np.array_equal(got_lab, exp_lab[:total])
    finally:
        plan.close()
        h.set_precision(H.PREC_FP32_EXACT)


def test_plan_clamps_capacity_and_index_changes(index):
    import torch
    h = index
    nq, k = 500, 10
    Q, hm, hkp, hef = _batch(3, nq, 6, 80)
    hm[7] = 40  # above m_max: runs with m_max and is reported
    q = torch.from_numpy(Q).cuda()
    m = torch.from_numpy(hm.astype(np.int32)).cuda()
    kp = torch.from_numpy(hkp.astype(np.int32)).cuda()
    ef = torch.from_numpy(hef.astype(np.int32)).cuda()
    off = torch.zeros(nq + 1, dtype=torch.int64, device="cuda")
    lab = torch.zeros(4, dtype=torch.int64, device="cuda")
    plan = h.search_plan(q.data_ptr(), nq, m.data_ptr(), kp.data_ptr(), ef.data_ptr(), 6, 80, 1.0, k,
                         off.data_ptr(), lab.data_ptr(), 4)
    try:
        torch.cuda.synchronize()
        plan.run()
        with pytest.raises(H.HrnnError) as e:  # far more than 4 results
            plan.result()
        assert e.value.code == H.ERR_CAPACITY
        assert int(off[-1].item()) > 4
        # the clamped query equals a batch call with m = m_max
        m_ref = m.clone()
        m_ref[7] = 6
        exp_off, _ = _regular(h, torch, q, m_ref, kp, ef, k, int(off[-1].item()) + 16)
        assert np.array_equal(off.cpu().numpy(), exp_off)
        h.setEf(50)  # any call that changes the index invalidates the plan
        with pytest.raises(H.HrnnError) as e:
            plan.run()
        assert e.value.code == H.ERR_STATE
    finally:
        plan.close()


def test_autotuned_launch_shape_keeps_answers(index):
    h = index
    Q, _, _, _ = _batch(4, 2048, 8, 120)
    h.set_autotune(False)
    plain = h.search_rknn_batch(Q, 5, 100, 150, threshold=1.0, k=10)
    st0 = h.last_search_stats()
    h.set_autotune(True)
    tuned = h.search_rknn_batch(Q, 5, 100, 150, threshold=1.0, k=10)
    st1 = h.last_search_stats()
    again = h.search_rknn_batch(Q, 5, 100, 150, threshold=1.0, k=10)  # the cached shape
    st2 = h.last_search_stats()
    assert (st1["a_warps_per_block"], st1["a_visit_slots"]) in {(w, v) for w in (2, 4) for v in (256, 512, 1024)}
    assert (st2["a_warps_per_block"], st2["a_visit_slots"]) == (st1["a_warps_per_block"], st1["a_visit_slots"])
    assert (st0["a_warps_per_block"], st0["a_visit_slots"]) == (4, 512)  # the untuned shape at d = 128
    for a, b, c in zip(plain, tuned, again):
        assert np.array_equal(a, b) and np.array_equal(a, c)
    assert st1["n_result"] == st0["n_result"]
