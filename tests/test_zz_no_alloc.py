"""hrnn_build_rknng_noalloc: the CSR transpose for callers that cannot allocate
device memory (an arena that owns every device byte, a serving loop that must not
call cudaMalloc).  Through the C ABI, with caller-owned device buffers, its output
must equal the allocating entry point's (hrnn_build_rknng + hrnn_get_rknng) on
two calls in a row -- integer output, so equal means bit-identical.

This file is collected last so that a failure here comes after every other test;
it also passes on its own in a fresh process."""
import numpy as np
import pytest

from oracle import idx

import hrnn_b200 as H

pytestmark = pytest.mark.gpu


def _graph_hubs(n=40000, K=48, seed=8):
    rng = np.random.default_rng(seed)
    ids = np.empty((n, K), np.uint32)
    for i in range(n):
        row = [h for h in range(3) if h != i]       # every list points at 3 hubs
        for j in rng.integers(0, n, size=K + 16):
            j = int(j)
            if j != i and j not in row:
                row.append(j)
        ids[i] = row[:K]
    cnt = rng.integers(K // 2, K + 1, size=n).astype(np.uint32)
    return ids, cnt


def _allocating_csr(tmp_path, ids, cnt, name):
    n, K = ids.shape
    X = np.zeros((n, 16), np.float32)
    d = np.sort(np.random.default_rng(1).random((n, K)).astype(np.float32), axis=1)
    p = str(tmp_path / name)
    idx.write_idx(p, X, ids, d, cnt, M=4)
    h = H.HRNN.load(p, 16)
    h.buildRKNNG()
    return h.get_rknng(reference_order=False)


def _noalloc_csr(ids, cnt):
    import torch
    n, K = ids.shape
    d_ids = torch.from_numpy(ids.view(np.int32)).cuda()
    d_cnt = torch.from_numpy(cnt.view(np.int32)).cuda()
    total = int(np.sum(cnt & 0xFFFF))
    d_off = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    d_ent = torch.zeros(total + 8, dtype=torch.int64, device="cuda")   # room for u64 entries
    torch.cuda.synchronize()
    rb, wide, ne = H.build_rknng_noalloc(d_ids.data_ptr(), d_cnt.data_ptr(), n, K, d_off.data_ptr(),
                                         d_ent.data_ptr(), total + 8)
    assert ne == total
    off = d_off.cpu().numpy().view(np.uint64)
    raw = d_ent.cpu().numpy().view(np.uint8)
    ent = raw.view(np.uint64)[:ne] if wide else raw.view(np.uint32)[:ne]
    return off, ent, rb, wide


def test_noalloc_matches_allocating_entry_point_twice(tmp_path, golden_idx):
    f = idx.read_idx(golden_idx)
    g_ids, _, g_cnt = f.knng()
    h_ids, h_cnt = _graph_hubs()
    exp_g = _allocating_csr(tmp_path, g_ids, g_cnt, "g.idx")
    exp_h = _allocating_csr(tmp_path, h_ids, h_cnt, "h.idx")
    # two calls in a row on different graphs, then the first graph again: the shared
    # scratch keeps the previous call's contents and must not leak into the next one
    for ids, cnt, exp in ((g_ids, g_cnt, exp_g), (h_ids, h_cnt, exp_h), (g_ids, g_cnt, exp_g)):
        off, ent, rb, wide = _noalloc_csr(ids, cnt)
        assert rb == exp[2] and wide == exp[3]
        assert np.array_equal(off, exp[0])
        assert np.array_equal(ent, exp[1])
    assert int(np.max(np.diff(exp_h[0]))) > 16384       # long lists took the staging path


def test_noalloc_rejects_sizes_beyond_its_scratch():
    fake = 256  # never dereferenced: the size check comes first
    with pytest.raises(H.HrnnError) as e:
        H.build_rknng_noalloc(fake, fake, (1 << 21) + 1, 8, fake, fake, 16)
    assert e.value.code == H.ERR_LIMIT and "2097152" in str(e.value)


def test_noalloc_rejects_a_graph_with_bad_ids_or_counts():
    """The caller's graph is checked on the device before anything is scattered:
    an id >= n, or a count above K, returns HRNN_ERR_ARG (no out-of-range write),
    and the next call on a valid graph still succeeds."""
    import torch
    n, K = 1000, 8
    rng = np.random.default_rng(3)
    ids = rng.integers(0, n, size=(n, K)).astype(np.uint32)
    cnt = np.full(n, K, np.uint32)
    for bad_ids, bad_cnt in ((True, False), (False, True)):
        i2, c2 = ids.copy(), cnt.copy()
        if bad_ids:
            i2[17, 3] = n + 5
        if bad_cnt:
            c2[400] = K + 1
        d_ids = torch.from_numpy(i2.view(np.int32)).cuda()
        d_cnt = torch.from_numpy(c2.view(np.int32)).cuda()
        d_off = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
        d_ent = torch.zeros(n * K + 8, dtype=torch.int64, device="cuda")
        with pytest.raises(H.HrnnError) as e:
            H.build_rknng_noalloc(d_ids.data_ptr(), d_cnt.data_ptr(), n, K, d_off.data_ptr(), d_ent.data_ptr(),
                                  n * K + 8)
        assert e.value.code == H.ERR_ARG
        assert ("id(s) >= n" in str(e.value)) and ("count(s) above K" in str(e.value))
    off, ent, rb, wide = _noalloc_csr(ids, cnt)
    assert int(off[-1]) == n * K and not wide


def test_noalloc_wide_entries():
    """node_bits + rank_bits > 32 gives u64 entries: n = 2^20 + 1 (21 node bits),
    K = 2049 (12 rank bits).  The n x K id array lives on the device (8.6 GB);
    most nodes list 0-3 neighbours, 64 nodes a full K, so ranks up to 2048 occur.
    Checked against a numpy transpose: segments in (rank, owner) order."""
    import torch
    n, K = (1 << 20) + 1, 2049
    g = torch.Generator(device="cuda").manual_seed(5)
    d_ids = torch.randint(0, n, (n, K), dtype=torch.int32, device="cuda", generator=g)
    rng = np.random.default_rng(6)
    cnt = rng.integers(0, 4, size=n).astype(np.uint32)
    full = rng.choice(n, 64, replace=False)
    cnt[full] = K
    d_cnt = torch.from_numpy(cnt.view(np.int32)).cuda()
    total = int(cnt.sum())
    d_off = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    d_ent = torch.zeros(total + 8, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    rb, wide, ne = H.build_rknng_noalloc(d_ids.data_ptr(), d_cnt.data_ptr(), n, K, d_off.data_ptr(),
                                         d_ent.data_ptr(), total + 8)
    assert (rb, wide, ne) == (12, True, total)
    # expected CSR from the used part of the graph
    head = d_ids[:, :3].cpu().numpy().view(np.uint32)
    rows = d_ids[torch.from_numpy(np.sort(full)).cuda()].cpu().numpy().view(np.uint32)
    own, rnk, tgt = [], [], []
    for j in range(3):
        sel = np.nonzero((cnt > j) & (cnt < K))[0]
        own.append(sel), rnk.append(np.full(len(sel), j)), tgt.append(head[sel, j])
    for r, i in enumerate(np.sort(full)):
        own.append(np.full(K, i)), rnk.append(np.arange(K)), tgt.append(rows[r])
    own, rnk, tgt = (np.concatenate(a).astype(np.uint64) for a in (own, rnk, tgt))
    order = np.lexsort((own, rnk, tgt))
    exp_ent = (own[order] << np.uint64(12)) | rnk[order]
    exp_off = np.zeros(n + 1, np.uint64)
    exp_off[1:] = np.cumsum(np.bincount(tgt.astype(np.int64), minlength=n))
    del d_ids
    off = d_off.cpu().numpy().view(np.uint64)
    ent = d_ent.cpu().numpy().view(np.uint64)[:ne]
    assert np.array_equal(off, exp_off)
    assert np.array_equal(ent, exp_ent)
