"""GPU parity of the exact-order L2 kernel, the reverse-CSR builder and the .idx
reader/writer, through the C ABI, against the reference's own outputs."""
import os

import numpy as np
import pytest

from conftest import golden_results, have_ref
from oracle import data, idx, port

import hrnn_b200 as H

pytestmark = pytest.mark.gpu


def test_l2_bit_exact_all_dims(golden_l2):
    for d in (7, 16, 20, 32, 36, 96, 128, 256):
        A, B, D = golden_l2[f"A_{d}"], golden_l2[f"B_{d}"], golden_l2[f"D_{d}"]
        got = H.l2_batch(A, B, lanes=16, fused=2)
        assert np.array_equal(got.view(np.uint32), D.view(np.uint32)), d


def test_l2_other_orders_match_oracle():
    rng = np.random.default_rng(9)
    for d in (16, 48, 128):
        A = rng.normal(0, 3, (300, d)).astype(np.float32)
        B = rng.normal(0, 3, (300, d)).astype(np.float32)
        for lanes in (16, 8, 4):
            for fused in (0, 1, 2, 3):
                g = H.l2_batch(A, B, lanes, fused)
                o = port.l2_batch(A, B, lanes, fused)
                assert np.array_equal(g.view(np.uint32), o.view(np.uint32)), (d, lanes, fused)


def test_idx_roundtrip_byte_exact(golden_idx, tmp_path):
    h = H.HRNN.load(golden_idx, 32)
    out = str(tmp_path / "rt.idx")
    h.saveIndex(out)
    assert open(out, "rb").read() == open(golden_idx, "rb").read()


def test_csr_rebuild_bit_exact(golden_idx, tmp_path):
    f = idx.read_idx(golden_idx)
    h = H.HRNN.load(golden_idx, 32)
    h.buildRKNNG()                     # device build replaces the loaded CSR
    off, ent, rb, wide = h.get_rknng(reference_order=False)
    ids, _, cnt = f.knng()
    o_off, o_ent, o_rb, o_wide = port.rknng(ids, cnt, f.n, f.K, canonical=True)
    assert rb == o_rb and wide == o_wide
    assert np.array_equal(off, o_off) and np.array_equal(ent, o_ent)
    # reference byte order (the std::sort call of buildRKNNG_fill, hrnn.h:1928-1934)
    off2, ent2, _, _ = h.get_rknng(reference_order=True)
    assert np.array_equal(off2, f.csr_offsets) and np.array_equal(ent2, f.csr_entries)
    out = str(tmp_path / "rebuilt.idx")
    h.saveIndex(out)
    assert open(out, "rb").read() == open(golden_idx, "rb").read()


def test_csr_large_random_graph_with_hubs(tmp_path):
    """A KNN graph with heavy hubs: segments far above the warp-sort size."""
    rng = np.random.default_rng(3)
    n, K, d = 30000, 64, 16
    X = rng.normal(size=(n, d)).astype(np.float32)
    ids = np.empty((n, K), np.uint32)
    for i in range(n):                         # distinct ids, never self, 8 slots on 5 hubs
        row = [h for h in range(5) if h != i][:4]
        while len(row) < K:
            j = int(rng.integers(0, n))
            if j != i and j not in row:
                row.append(j)
        ids[i] = row
    cnt = rng.integers(K // 2, K + 1, size=n).astype(np.uint32)
    dists = np.sort(rng.random((n, K)).astype(np.float32), axis=1)
    p = str(tmp_path / "hubs.idx")
    idx.write_idx(p, X, ids, dists, cnt, M=4)
    h = H.HRNN.load(p, d)
    h.buildRKNNG()
    off, ent, rb, wide = h.get_rknng()
    o_off, o_ent, _, _ = port.rknng(ids, cnt, n, K, canonical=True)
    assert np.array_equal(off, o_off) and np.array_equal(ent, o_ent)
    assert int(np.max(np.diff(off))) > 16384          # exercised the global-memory sort


def test_wide_entries_match_narrow_and_reference(golden_idx, tmp_path, monkeypatch):
    """64-bit reverse-CSR entries (forced on a small index with HRNN_RKNNG_WIDE=1,
    the layout an index with node_bits + rank_bits > 32 gets): the same offsets and
    (owner, rank) values as the 32-bit ones, the same search answers, and a saved
    wide .idx that the reference loads and answers identically."""
    h = H.HRNN.load(golden_idx, 32)
    Q = data.mixture(64, 32, 12, 1.0, 11, 77)
    monkeypatch.delenv("HRNN_RKNNG_WIDE", raising=False)
    h.buildRKNNG()  # the loaded CSR is in the file's (reference) order; rebuild both in the device's
    narrow = h.search_rknn_batch(Q, 10, 24, 40, threshold=1.0, k=10)
    off_n, ent_n, rb_n, wide_n = h.get_rknng()
    monkeypatch.setenv("HRNN_RKNNG_WIDE", "1")
    h.buildRKNNG()
    off_w, ent_w, rb_w, wide_w = h.get_rknng()
    assert wide_w and not wide_n and rb_w == rb_n
    assert ent_w.dtype == np.uint64 and ent_n.dtype == np.uint32
    assert np.array_equal(off_w, off_n) and np.array_equal(ent_w, ent_n.astype(np.uint64))
    wide = h.search_rknn_batch(Q, 10, 24, 40, threshold=1.0, k=10)
    assert all(np.array_equal(a, b) for a, b in zip(narrow, wide))
    exp = port.OracleIndex(idx.read_idx(golden_idx)).search_batch(Q, 10, 24, 40, threshold=1.0, k=10)
    assert all(np.array_equal(a, b) for a, b in zip(wide, exp))
    if have_ref():
        from oracle import ref
        p = str(tmp_path / "wide.idx")
        h.saveIndex(p)
        r = ref.RefIndex.load(p, 32)
        a = r.search_batch(Q, 10, 24, 40, threshold=1.0, k=10)
        assert all(np.array_equal(x, y) for x, y in zip(a, wide))
