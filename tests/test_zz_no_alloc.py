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
