"""ctypes bindings of liboracle.so, the C restatement (test infrastructure only)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .idx import IdxFile

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(os.path.join(_HERE, "liboracle.so"))
        _lib.orc_l2.restype = C.c_float
        _lib.orc_l2.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_int]
        _lib.orc_rknng_params.restype = C.c_uint32
        _lib.orc_search_rknn.restype = C.c_size_t
        _lib.orc_search_rknn_batch.restype = C.c_int
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class OrcIndex(C.Structure):
    _fields_ = [
        ("n", C.c_size_t), ("d", C.c_size_t), ("maxM0", C.c_size_t), ("maxM", C.c_size_t),
        ("K", C.c_size_t),
        ("vec", C.c_void_p), ("adj0", C.c_void_p), ("level", C.c_void_p),
        ("upper_off", C.c_void_p), ("upper", C.c_void_p),
        ("enterpoint", C.c_uint32), ("maxlevel", C.c_int32),
        ("knn_cnt", C.c_void_p), ("knn_dist", C.c_void_p),
        ("kdist_serve", C.c_void_p), ("max_k_serve", C.c_size_t),
        ("csr_off", C.c_void_p), ("csr_ent", C.c_void_p), ("entry_bytes", C.c_int),
        ("rank_bits", C.c_uint32), ("labels", C.c_void_p), ("lanes", C.c_int), ("fused", C.c_int),
    ]


class OrcStats(C.Structure):
    _fields_ = [(f, C.c_uint64) for f in
                ("n_dist", "n_expanded", "n_posting", "n_cand", "n_verified", "n_result")]


def l2(a: np.ndarray, b: np.ndarray, lanes: int = 16, fused: int = 2) -> float:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return float(lib().orc_l2(_p(a), _p(b), a.size, lanes, fused))


def l2_batch(A: np.ndarray, B: np.ndarray, lanes: int = 16, fused: int = 2) -> np.ndarray:
    A = np.ascontiguousarray(A, np.float32)
    B = np.ascontiguousarray(B, np.float32)
    out = np.empty(A.shape[0], np.float32)
    lib().orc_l2_batch(_p(A), _p(B), C.c_size_t(A.shape[0]), C.c_size_t(A.shape[1]), lanes, fused,
                       _p(out))
    return out


class OracleIndex:
    """Holds numpy arrays of an index and the C view over them."""

    def __init__(self, f: IdxFile, lanes: int = 16, fused: int = 2, max_k_serve: int = 0):
        self.f = f
        self.vec = np.ascontiguousarray(f.vectors())
        self.adj0 = np.ascontiguousarray(f.adj0())
        self.level = f.levels()
        self.upper_off, self.upper = f.upper()
        self.knn_ids, self.knn_dist, self.knn_cnt = f.knng()
        self.labels = np.ascontiguousarray(f.labels())
        self.kdist_serve = None
        if max_k_serve:
            j = np.arange(max_k_serve)[None, :]
            ks = np.where(j < self.knn_cnt[:, None], self.knn_dist[:, :max_k_serve],
                          np.float32(np.finfo(np.float32).max))
            self.kdist_serve = np.ascontiguousarray(ks, dtype=np.float32)
        s = OrcIndex()
        s.n, s.d, s.maxM0, s.maxM, s.K = f.n, f.dim, f.maxM0, f.maxM, f.K
        s.vec, s.adj0, s.level = _p(self.vec), _p(self.adj0), _p(self.level)
        s.upper_off, s.upper = _p(self.upper_off), _p(self.upper)
        s.enterpoint, s.maxlevel = f.enterpoint, f.maxlevel
        s.knn_cnt, s.knn_dist = _p(self.knn_cnt), _p(self.knn_dist)
        s.kdist_serve = _p(self.kdist_serve) if self.kdist_serve is not None else None
        s.max_k_serve = max_k_serve
        if f.rknng_built:
            self.csr_off = np.ascontiguousarray(f.csr_offsets)
            self.csr_ent = np.ascontiguousarray(f.csr_entries)
            s.csr_off, s.csr_ent = _p(self.csr_off), _p(self.csr_ent)
            s.entry_bytes, s.rank_bits = f.entry_bytes, f.rank_bits
        s.labels, s.lanes, s.fused = _p(self.labels), lanes, fused
        self.s = s

    def search_batch(self, Q, m, Kp, ef, threshold=1.0, k=10, threads=1):
        Q = np.ascontiguousarray(Q, np.float32)
        nq = Q.shape[0]
        m = np.ascontiguousarray(np.broadcast_to(np.asarray(m, np.uint32), (nq,)))
        Kp = np.ascontiguousarray(np.broadcast_to(np.asarray(Kp, np.uint32), (nq,)))
        ef = np.ascontiguousarray(np.broadcast_to(np.asarray(ef, np.uint32), (nq,)))
        off = np.zeros(nq + 1, np.uint64)
        cap = int(np.sum(m.astype(np.int64) * np.maximum(Kp, 1))) + 16
        lab = np.zeros(cap, np.uint64)
        rc = lib().orc_search_rknn_batch(C.byref(self.s), _p(Q), C.c_size_t(nq), _p(m), _p(Kp), _p(ef),
                                         C.c_float(threshold), C.c_uint32(k), _p(off), _p(lab),
                                         C.c_size_t(cap), threads)
        if rc == 2:
            cap = int(off[-1])
            lab = np.zeros(cap, np.uint64)
            rc = lib().orc_search_rknn_batch(C.byref(self.s), _p(Q), C.c_size_t(nq), _p(m), _p(Kp),
                                             _p(ef), C.c_float(threshold), C.c_uint32(k), _p(off),
                                             _p(lab), C.c_size_t(cap), threads)
        assert rc == 0
        return [lab[off[i]:off[i + 1]].copy() for i in range(nq)]

    def search_one(self, q, m, Kp, ef, threshold=1.0, k=10):
        """One query; returns (labels, proxies ascending by distance, stats dict)."""
        q = np.ascontiguousarray(q, np.float32)
        cap = max(1, m * max(Kp, 1)) + 16
        out = np.zeros(cap, np.uint64)
        score = np.zeros(self.f.n, np.float32)
        st = OrcStats()
        prox = np.zeros(max(m, 1), np.uint32)
        npx = C.c_size_t(0)
        r = lib().orc_search_rknn(C.byref(self.s), _p(q), C.c_size_t(m), C.c_float(threshold),
                                  C.c_size_t(k), C.c_size_t(Kp), C.c_size_t(ef), _p(out),
                                  C.c_size_t(cap), _p(score), C.byref(st), _p(prox), C.byref(npx))
        if r > cap:
            out = np.zeros(r, np.uint64)
            lib().orc_search_rknn(C.byref(self.s), _p(q), C.c_size_t(m), C.c_float(threshold),
                                  C.c_size_t(k), C.c_size_t(Kp), C.c_size_t(ef), _p(out),
                                  C.c_size_t(r), _p(score), None, None, None)
        stats = {f: getattr(st, f) for f, _ in OrcStats._fields_}
        return out[:r].copy(), prox[: npx.value].copy(), stats


def rknng(knn_ids, knn_cnt, n, K, canonical=True):
    """(offsets, entries, rank_bits, wide) of the reverse CSR (hrnn.h:1869-1935)."""
    wide = C.c_int(0)
    rb = lib().orc_rknng_params(C.c_size_t(n), C.c_size_t(K), C.byref(wide))
    ids = np.ascontiguousarray(knn_ids, np.uint32)
    cnt = np.ascontiguousarray(knn_cnt, np.uint32)
    off = np.zeros(n + 1, np.uint64)
    total = int(np.sum(cnt & 0xFFFF))
    ent = np.zeros(max(total, 1), np.uint64 if wide.value else np.uint32)
    lib().orc_rknng_presort(C.c_size_t(n), C.c_size_t(K), _p(ids), _p(cnt), C.c_uint32(rb),
                            wide.value, _p(off), _p(ent))
    if canonical:
        lib().orc_rknng_canonical(C.c_size_t(n), C.c_uint32(rb), wide.value, _p(off), _p(ent))
    return off, ent[:total], int(rb), bool(wide.value)


def refine(vec, ids, dists, cnt, is_new, iters, sample, lanes=16, fused=2):
    """Single-thread NNDescent (hrnn.h:1725-1862); arrays are updated in place."""
    n, K = ids.shape
    d = vec.shape[1]
    upd = np.zeros(max(iters, 1), np.uint64)
    jd = np.zeros(max(iters, 1), np.uint64)
    lib().orc_refine_knng(C.c_size_t(n), C.c_size_t(d), C.c_size_t(K), _p(vec), lanes, fused, _p(ids),
                          _p(dists), _p(cnt), _p(is_new), iters, sample, _p(upd), _p(jd))
    return upd[:iters], jd[:iters]
