"""The .idx loader range-checks every id the device kernels follow before it
uploads anything they read: a corrupt file is rejected with HRNN_ERR_FORMAT
instead of becoming out-of-bounds device reads in the search and refinement
kernels.  The corrupt files are made on the host from the reference-built golden
index (tests/golden/small_index.idx.gz) by changing single fields of its layout
(saveIndex, hrnn.h:861-927); the untouched file must still load."""
import struct

import numpy as np
import pytest

from oracle import idx

import hrnn_b200 as H

pytestmark = pytest.mark.gpu


def _layout(raw: bytes):
    f = idx.read_idx_bytes(raw)
    pos = idx._HDR.size
    l0 = pos
    pos += f.n * f.size_data_per_element
    upper_pos = []
    for i in range(f.n):
        (s,) = struct.unpack_from("<I", raw, pos)
        upper_pos.append(pos + 4)
        pos += 4 + s
    csr = pos
    return f, l0, upper_pos, csr


def _load_expect_format(tmp_path, raw: bytes, name: str):
    p = tmp_path / name
    p.write_bytes(raw)
    with pytest.raises(H.HrnnError) as e:
        H.HRNN.load(str(p), 32)
    assert e.value.code == H.ERR_FORMAT, str(e.value)
    return str(e.value)


def _put_u32(b: bytearray, off: int, v: int):
    struct.pack_into("<I", b, off, v & 0xFFFFFFFF)


def test_corrupt_ids_are_rejected(tmp_path, golden_idx):
    raw = open(golden_idx, "rb").read()
    f, l0, upper_pos, csr = _layout(raw)
    n, S = f.n, f.size_data_per_element
    h = H.HRNN.load(golden_idx, 32)  # the untouched file loads
    assert h.getCurrentElementCount() == n
    del h
    adj = f.adj0()
    e = int(np.nonzero((adj[:, 0] & 0xFFFF) >= 2)[0][0])
    rec = l0 + e * S

    b = bytearray(raw)
    _put_u32(b, rec + f.offsetLevel0 + 4 * 2, n + 7)            # level-0 link id >= cur
    assert "level-0" in _load_expect_format(tmp_path, bytes(b), "l0id.idx")
    b = bytearray(raw)
    _put_u32(b, rec + f.offsetLevel0, f.maxM0 + 1)               # level-0 count > maxM0
    assert "level-0" in _load_expect_format(tmp_path, bytes(b), "l0cnt.idx")

    ids, _, cnt = f.knng()
    e2 = int(np.nonzero(cnt >= 3)[0][0])
    rec2 = l0 + e2 * S
    b = bytearray(raw)
    _put_u32(b, rec2 + f.offsetKNNG + 4 + 8 * 1, n)             # KNN id >= cur
    assert "KNN" in _load_expect_format(tmp_path, bytes(b), "knnid.idx")
    b = bytearray(raw)
    _put_u32(b, rec2 + f.offsetKNNG, f.K + 1)                   # KNN count > K
    assert "KNN" in _load_expect_format(tmp_path, bytes(b), "knncnt.idx")

    lv = f.levels()
    e3 = next(i for i in range(n) if lv[i] >= 1 and struct.unpack_from("<I", raw, upper_pos[i])[0] & 0xFFFF >= 1)
    b = bytearray(raw)
    _put_u32(b, upper_pos[e3] + 4, n + 1)                        # upper-layer id >= cur
    assert "upper-layer" in _load_expect_format(tmp_path, bytes(b), "upid.idx")
    low = int(np.nonzero(lv == 0)[0][0])
    b = bytearray(raw)
    _put_u32(b, upper_pos[e3] + 4, low)                          # level-1 link to a level-0 element
    assert "upper-layer" in _load_expect_format(tmp_path, bytes(b), "uplevel.idx")

    b = bytearray(raw)
    ep_off = struct.calcsize("<IQQQQQQi")                        # enterpoint follows maxlevel
    _put_u32(b, ep_off, n + 3)
    assert "entry point" in _load_expect_format(tmp_path, bytes(b), "ep.idx")

    assert f.rknng_built
    eb = f.entry_bytes
    ent0 = csr + 1 + 4 + 8 + 8 * (n + 1) + 8
    b = bytearray(raw)
    if eb == 4:
        _put_u32(b, ent0, (n + 2) << f.rank_bits)                # CSR owner >= cur
    else:
        struct.pack_into("<Q", b, ent0, (n + 2) << f.rank_bits)
    assert "reverse CSR" in _load_expect_format(tmp_path, bytes(b), "csrown.idx")
    b = bytearray(raw)
    offs0 = csr + 1 + 4 + 8
    struct.pack_into("<Q", b, offs0 + 8 * 5, int(f.csr_offsets[5]) + 10 ** 6)  # offsets not ascending
    assert "reverse CSR" in _load_expect_format(tmp_path, bytes(b), "csroff.idx")
    if (1 << f.rank_bits) > f.K:
        b = bytearray(raw)
        v = int(f.csr_entries[0])
        v = (v >> f.rank_bits << f.rank_bits) | f.K                # rank = K (a slot that does not exist)
        if eb == 4:
            _put_u32(b, ent0, v)
        else:
            struct.pack_into("<Q", b, ent0, v)
        assert "reverse CSR" in _load_expect_format(tmp_path, bytes(b), "csrrank.idx")
