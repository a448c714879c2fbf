"""Independent numpy reader of the reference's .idx file (test infrastructure).

Layout restated from saveIndex / loadIndex (include/hnswlib/hrnn.h:861-1047):
a POD header (magic 0x4E4E5248 ... rknng_built), the level-0 blob of
cur_element_count x size_data_per_element bytes, one (u32 size, bytes) record per
element for the upper layers, then -- when rknng_built -- the reverse CSR.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

MAGIC = 0x4E4E5248
_HDR = struct.Struct("<IQQQQQQiIQQQdQQQQ??")  # hrnn.h:868-890


@dataclass
class IdxFile:
    offsetLevel0: int
    max_elements: int
    n: int
    size_data_per_element: int
    label_offset: int
    offsetData: int
    maxlevel: int
    enterpoint: int
    maxM: int
    maxM0: int
    M: int
    mult: float
    ef_construction: int
    K: int
    size_knng_slot: int
    offsetKNNG: int
    knng_built: bool
    rknng_built: bool
    level0: np.ndarray = field(repr=False)          # (n, size_data_per_element) u8
    link_sizes: np.ndarray = field(repr=False)      # (n,) u32 bytes of upper-layer blob
    upper_blobs: list = field(repr=False)           # per element bytes
    entry_bytes: int = 0
    rank_bits: int = 0
    csr_offsets: np.ndarray | None = field(default=None, repr=False)
    csr_entries: np.ndarray | None = field(default=None, repr=False)
    rank_mask: int = 0

    # ---- derived views ------------------------------------------------------
    @property
    def dim(self) -> int:
        return (self.label_offset - self.offsetData) // 4

    def adj0(self) -> np.ndarray:
        w = 1 + self.maxM0
        return np.ascontiguousarray(self.level0[:, : 4 * w]).view(np.uint32).reshape(self.n, w)

    def vectors(self) -> np.ndarray:
        b = self.level0[:, self.offsetData : self.offsetData + 4 * self.dim]
        return np.ascontiguousarray(b).view(np.float32).reshape(self.n, self.dim)

    def labels(self) -> np.ndarray:
        b = self.level0[:, self.label_offset : self.label_offset + 8]
        return np.ascontiguousarray(b).view(np.uint64).reshape(self.n)

    def knng(self):
        """(ids (n,K) u32, dists (n,K) f32, cnt (n,) u32 -- low 16 bits)."""
        K = self.K
        o = self.offsetKNNG
        cntw = np.ascontiguousarray(self.level0[:, o : o + 4]).view(np.uint32).reshape(self.n)
        pairs = np.ascontiguousarray(self.level0[:, o + 4 : o + 4 + 8 * K]).view(np.uint32)
        pairs = pairs.reshape(self.n, K, 2)
        ids = np.ascontiguousarray(pairs[:, :, 0])
        dists = np.ascontiguousarray(pairs[:, :, 1]).view(np.float32)
        return ids, dists, (cntw & 0xFFFF).astype(np.uint32)

    def levels(self) -> np.ndarray:
        per = 4 * (self.maxM + 1)
        return (self.link_sizes // per).astype(np.int32)

    def upper(self):
        """(upper_off (n,) u64 word offsets, upper (W,) u32) -- level l block of
        element i starts at upper_off[i] + (l-1)*(1+maxM)."""
        off = np.zeros(self.n, dtype=np.uint64)
        parts = []
        pos = 0
        for i, b in enumerate(self.upper_blobs):
            off[i] = pos
            if b:
                a = np.frombuffer(b, dtype=np.uint32)
                parts.append(a)
                pos += a.size
        up = np.concatenate(parts) if parts else np.zeros(1, dtype=np.uint32)
        return off, np.ascontiguousarray(up)


def read_idx(path: str) -> IdxFile:
    with open(path, "rb") as f:
        return read_idx_bytes(f.read())


def read_idx_bytes(raw: bytes) -> IdxFile:
    h = _HDR.unpack_from(raw, 0)
    if h[0] != MAGIC:
        raise ValueError("Not an HRNN index file (bad magic)")
    pos = _HDR.size
    (_, offL0, maxel, n, sz, labo, offd, maxlevel, ep, maxM, maxM0, M, mult, efc, K, slot,
     offK, kb, rb) = h
    level0 = np.frombuffer(raw, dtype=np.uint8, count=n * sz, offset=pos).reshape(n, sz)
    pos += n * sz
    sizes = np.zeros(n, dtype=np.uint32)
    blobs = []
    for i in range(n):
        (s,) = struct.unpack_from("<I", raw, pos)
        pos += 4
        sizes[i] = s
        blobs.append(raw[pos : pos + s] if s else b"")
        pos += s
    f = IdxFile(offL0, maxel, n, sz, labo, offd, maxlevel, ep, maxM, maxM0, M, mult, efc, K, slot,
                offK, kb, rb, level0, sizes, blobs)
    if rb:
        (eb,) = struct.unpack_from("<B", raw, pos); pos += 1
        (rbits,) = struct.unpack_from("<I", raw, pos); pos += 4
        (no,) = struct.unpack_from("<Q", raw, pos); pos += 8
        offs = np.frombuffer(raw, dtype=np.uint64, count=no, offset=pos); pos += 8 * no
        (ne,) = struct.unpack_from("<Q", raw, pos); pos += 8
        dt = np.uint64 if eb == 8 else np.uint32
        ents = np.frombuffer(raw, dtype=dt, count=ne, offset=pos); pos += eb * ne
        (mask,) = struct.unpack_from("<Q" if eb == 8 else "<I", raw, pos)
        f.entry_bytes, f.rank_bits, f.csr_offsets, f.csr_entries, f.rank_mask = eb, rbits, offs, ents, mask
    return f


def write_idx(path: str, X: np.ndarray, knn_ids: np.ndarray, knn_dists: np.ndarray, knn_cnt: np.ndarray,
              M: int = 4, adj0: np.ndarray | None = None, labels: np.ndarray | None = None,
              knng_built: bool = True) -> None:
    """Writes a single-layer index in the reference's layout (test fixtures only):
    level-0 links from adj0 ((n, 1+2M) u32, default empty), the given KNN slot,
    no upper layers, no reverse CSR."""
    n, d = X.shape
    K = knn_ids.shape[1]
    maxM0 = 2 * M
    links = 4 * (1 + maxM0)
    offK, slot = links, 4 + 8 * K
    offD = offK + slot
    labo = offD + 4 * d
    sz = labo + 8
    rec = np.zeros((n, sz), np.uint8)
    if adj0 is not None:
        rec[:, :links] = np.ascontiguousarray(adj0, np.uint32).view(np.uint8).reshape(n, links)
    rec[:, offK:offK + 4] = np.ascontiguousarray(knn_cnt, np.uint32).view(np.uint8).reshape(n, 4)
    pairs = np.empty((n, K, 2), np.uint32)
    pairs[:, :, 0] = knn_ids
    pairs[:, :, 1] = np.ascontiguousarray(knn_dists, np.float32).view(np.uint32)
    rec[:, offK + 4:offK + slot] = pairs.view(np.uint8).reshape(n, 8 * K)
    rec[:, offD:labo] = np.ascontiguousarray(X, np.float32).view(np.uint8).reshape(n, 4 * d)
    lab = np.arange(n, dtype=np.uint64) if labels is None else np.asarray(labels, np.uint64)
    rec[:, labo:sz] = lab.view(np.uint8).reshape(n, 8)
    hdr = _HDR.pack(MAGIC, 0, n, n, sz, labo, offD, 0, 0, M, maxM0, M, 1.0 / np.log(M), 100, K, slot, offK,
                    knng_built, False)
    with open(path, "wb") as f:
        f.write(hdr)
        f.write(rec.tobytes())
        f.write(np.zeros(n, np.uint32).tobytes())
