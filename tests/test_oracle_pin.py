"""Pins the oracle (the C restatement in oracle/hrnn_oracle.c) against outputs of
the reference itself: the committed golden fixtures, and -- where oracle/_ref is
built -- the reference compiled from its sources on fresh seeded inputs."""
import numpy as np
import pytest

from conftest import golden_results, have_ref
from oracle import data, idx, port


def test_l2_matches_reference_all_dims(golden_l2):
    for d in (7, 16, 20, 32, 36, 96, 128, 256):
        A, B, D = golden_l2[f"A_{d}"], golden_l2[f"B_{d}"], golden_l2[f"D_{d}"]
        got = port.l2_batch(A, B, lanes=16, fused=2)
        assert np.array_equal(got.view(np.uint32), D.view(np.uint32)), d


def test_l2_order_matters(golden_l2):
    # A different summation order gives different bits on some pairs: the pin is real.
    A, B, D = golden_l2["A_128"], golden_l2["B_128"], golden_l2["D_128"]
    for lanes, fused in ((16, 3), (8, 2), (4, 2)):
        got = port.l2_batch(A, B, lanes=lanes, fused=fused)
        assert not np.array_equal(got.view(np.uint32), D.view(np.uint32))


def test_idx_reader(golden_idx):
    f = idx.read_idx(golden_idx)
    assert (f.n, f.dim, f.K, f.maxM0, f.maxM) == (1500, 32, 24, 16, 8)
    assert f.knng_built and f.rknng_built and f.entry_bytes == 4
    ids, dists, cnt = f.knng()
    assert np.all(cnt <= 24) and np.all(np.diff(dists[cnt == 24], axis=1) >= 0)


def test_search_matches_reference(golden_idx, golden_search):
    O = port.OracleIndex(idx.read_idx(golden_idx))
    Q = golden_search["Q"]
    for i, (m, kp, ef, th, k) in enumerate(golden_search["sweep"]):
        got = O.search_batch(Q, int(m), int(kp), int(ef), threshold=float(th), k=int(k))
        exp = golden_results(golden_search, i)
        for q in range(len(Q)):
            assert np.array_equal(got[q], exp[q]), (i, q)


def test_csr_matches_reference(golden_idx):
    f = idx.read_idx(golden_idx)
    ids, _, cnt = f.knng()
    off, ent, rb, wide = port.rknng(ids, cnt, f.n, f.K, canonical=True)
    assert rb == f.rank_bits and not wide
    assert np.array_equal(off, f.csr_offsets)
    mask = (1 << rb) - 1
    ref_ent = f.csr_entries
    for b in range(f.n):
        s = slice(int(off[b]), int(off[b + 1]))
        r = ref_ent[s]
        assert np.array_equal(r & mask, np.sort(r & mask))            # reference: rank-sorted
        key = (r & mask).astype(np.uint64) << 32 | (r >> rb).astype(np.uint64)
        assert np.array_equal(ent[s], r[np.argsort(key, kind="stable")])  # same entries


def test_refine_matches_single_thread_reference(golden_refine):
    g = golden_refine
    ids, dists, cnt = g["pre_ids"].copy(), g["pre_dists"].copy(), g["pre_cnt"].copy()
    is_new = (np.arange(ids.shape[1])[None, :] < cnt[:, None]).astype(np.uint8)
    port.refine(g["X"], ids, dists, cnt, is_new, int(g["iters"]), int(g["sample"]))
    assert np.array_equal(cnt, g["post_cnt"])
    for i in range(len(cnt)):
        c = int(cnt[i])
        assert np.array_equal(ids[i, :c], g["post_ids"][i, :c]), i
        assert np.array_equal(dists[i, :c].view(np.uint32), g["post_dists"][i, :c].view(np.uint32)), i


@pytest.mark.skipif(not have_ref(), reason="reference library oracle/_ref not built")
def test_oracle_vs_live_reference(tmp_path):
    from oracle import ref
    X = data.mixture(4000, 48, 16, 1.0, 3, 3)
    Q = data.mixture(150, 48, 16, 1.0, 3, 4)
    r = ref.RefIndex.create(48, 4000, 12, 80, 100, 40)
    r.add_points(X, threads=4)
    r.refine(2, 16, threads=4)
    r.build_rknng()
    p = str(tmp_path / "r.idx")
    r.save(p)
    O = port.OracleIndex(idx.read_idx(p))
    for m, kp, ef, th, k in ((1, 40, 20, 1.0, 10), (6, 20, 50, 1.0, 10), (15, 40, 30, 2.0, 7)):
        a = r.search_batch(Q, m, kp, ef, threshold=th, k=k)
        b = O.search_batch(Q, m, kp, ef, threshold=th, k=k)
        assert all(np.array_equal(x, y) for x, y in zip(a, b))


def test_budget_mlp_oracle_finite_differences():
    """The FP64 budget-MLP oracle's analytic gradients against central differences."""
    from oracle import mlp
    rng = np.random.default_rng(7)
    params = [p.astype(np.float64) for p in mlp.init_params(3)]
    X = rng.standard_normal((6, 256)).astype(np.float32)
    Y = rng.integers(0, 2, (6, 2)).astype(np.uint8)
    _, grads = mlp.loss_and_grads(params, X, Y, bf16_ops=False)
    h = 1e-6
    for t, idxs in ((0, [(0, 0), (17, 200)]), (1, [(5,)]), (2, [(3, 9), (255, 1)]), (3, [(100,)]),
                    (4, [(0, 7), (1, 255)]), (5, [(0,), (1,)])):
        for ix in idxs:
            pp = [p.copy() for p in params]
            pp[t][ix] += h
            lp = mlp.loss_of(mlp.forward(pp, X, bf16_ops=False)[4], Y)
            pp[t][ix] -= 2 * h
            lm = mlp.loss_of(mlp.forward(pp, X, bf16_ops=False)[4], Y)
            num = (lp - lm) / (2 * h)
            assert abs(num - grads[t][ix]) <= 1e-6 + 1e-5 * abs(num), (t, ix, num, grads[t][ix])


def test_bf16_rounding_oracle():
    from oracle import mlp
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1.0 + 2 ** -9], np.float32)
    assert np.array_equal(mlp.bf16(x), [1.0, 1.0, 1.0 + 4 * 2 ** -8, -2.5, 1.0])
