"""ctypes bindings of _ref/libhrnn_ref.so: the reference's own hrnn.h compiled from
its sources by oracle/Makefile (test infrastructure only)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(_HERE, "_ref", "libhrnn_ref.so")
_lib = None


def available() -> bool:
    return os.path.exists(PATH)


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(PATH)
        for f in ("ref_create", "ref_load"):
            getattr(_lib, f).restype = C.c_void_p
        _lib.ref_create.argtypes = [C.c_size_t] * 6
        _lib.ref_load.argtypes = [C.c_char_p, C.c_size_t, C.c_size_t]
        _lib.ref_l2.restype = C.c_float
        _lib.ref_l2.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        _lib.ref_count.restype = C.c_size_t
        _lib.ref_count.argtypes = [C.c_void_p]
        _lib.ref_last_error.restype = C.c_char_p
        _lib.ref_free.argtypes = [C.c_void_p]
        for f in ("ref_add_points", "ref_refine", "ref_build_rknng", "ref_build_mutable",
                  "ref_insert_dynamic", "ref_save", "ref_compact", "ref_search_batch",
                  "ref_get_csr"):
            getattr(_lib, f).restype = C.c_int
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _check(rc):
    if rc:
        raise RuntimeError(lib().ref_last_error().decode())


def l2(a, b) -> float:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return float(lib().ref_l2(_p(a), _p(b), a.size))


def l2_batch(A, B) -> np.ndarray:
    A = np.ascontiguousarray(A, np.float32)
    B = np.ascontiguousarray(B, np.float32)
    out = np.empty(A.shape[0], np.float32)
    lib().ref_l2_batch(_p(A), _p(B), C.c_size_t(A.shape[0]), C.c_size_t(A.shape[1]), _p(out))
    return out


class RefIndex:
    """The reference's HRNN<float> behind its own public methods."""

    def __init__(self, h, dim):
        if not h:
            raise RuntimeError(lib().ref_last_error().decode())
        self.h = C.c_void_p(h)
        self.dim = dim

    @classmethod
    def create(cls, dim, max_elements, M=16, ef_c=200, seed=100, K=100):
        return cls(lib().ref_create(dim, max_elements, M, ef_c, seed, K), dim)

    @classmethod
    def load(cls, path, dim, max_elements=0):
        return cls(lib().ref_load(path.encode(), dim, max_elements), dim)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.ref_free(self.h)
            self.h = None

    def add_points(self, X, labels=None, threads=1):
        X = np.ascontiguousarray(X, np.float32)
        labels = np.arange(len(X), dtype=np.uint64) if labels is None else np.ascontiguousarray(labels, np.uint64)
        _check(lib().ref_add_points(self.h, _p(X), C.c_size_t(len(X)), _p(labels), threads))

    def refine(self, iters, sample, threads=1):
        _check(lib().ref_refine(self.h, iters, sample, threads))

    def build_rknng(self):
        _check(lib().ref_build_rknng(self.h))

    def build_mutable(self):
        _check(lib().ref_build_mutable(self.h))

    def insert_dynamic(self, X, labels, m_update=0, bidirectional=False, threads=1):
        X = np.ascontiguousarray(X, np.float32)
        labels = np.ascontiguousarray(labels, np.uint64)
        _check(lib().ref_insert_dynamic(self.h, _p(X), C.c_size_t(len(X)), _p(labels),
                                        C.c_uint(m_update), int(bidirectional), threads))

    def save(self, path):
        _check(lib().ref_save(self.h, path.encode()))

    def compact(self, max_k_serve):
        _check(lib().ref_compact(self.h, C.c_size_t(max_k_serve)))

    def count(self):
        return lib().ref_count(self.h)

    def search_batch(self, Q, m, Kp, ef, threshold=1.0, k=10, threads=1, return_seconds=False):
        Q = np.ascontiguousarray(Q, np.float32)
        nq = Q.shape[0]
        m = np.ascontiguousarray(np.broadcast_to(np.asarray(m, np.uint32), (nq,)))
        Kp = np.ascontiguousarray(np.broadcast_to(np.asarray(Kp, np.uint32), (nq,)))
        ef = np.ascontiguousarray(np.broadcast_to(np.asarray(ef, np.uint32), (nq,)))
        off = np.zeros(nq + 1, np.uint64)
        cap = int(np.sum(m.astype(np.int64) * np.maximum(Kp, 1))) + 16
        lab = np.zeros(cap, np.uint64)
        secs = C.c_double(0)
        args = (self.h, _p(Q), C.c_size_t(nq), _p(m), _p(Kp), _p(ef), C.c_float(threshold),
                C.c_uint32(k), _p(off), _p(lab))
        rc = lib().ref_search_batch(*args, C.c_size_t(cap), threads, C.byref(secs))
        if rc == 2:
            lab = np.zeros(int(off[-1]), np.uint64)
            args = args[:-1] + (_p(lab),)
            rc = lib().ref_search_batch(*args, C.c_size_t(len(lab)), threads, C.byref(secs))
        _check(rc)
        res = [lab[off[i]:off[i + 1]].copy() for i in range(nq)]
        return (res, secs.value) if return_seconds else res

    def knng(self, K):
        n = self.count()
        ids = np.zeros((n, K), np.uint32)
        d = np.zeros((n, K), np.float32)
        cnt = np.zeros(n, np.uint32)
        lib().ref_get_knng(self.h, _p(ids), _p(d), _p(cnt))
        return ids, d, cnt

    def set_knng(self, ids, dists, cnt):
        ids = np.ascontiguousarray(ids, np.uint32)
        dists = np.ascontiguousarray(dists, np.float32)
        cnt = np.ascontiguousarray(cnt, np.uint32)
        lib().ref_set_knng(self.h, _p(ids), _p(dists), _p(cnt))

    def csr(self):
        no, ne = C.c_uint64(0), C.c_uint64(0)
        eb, rb = C.c_uint32(0), C.c_uint32(0)
        if lib().ref_get_csr(self.h, C.byref(no), C.byref(ne), C.byref(eb), C.byref(rb), None, None):
            raise RuntimeError("RKNNG not built")
        off = np.zeros(no.value, np.uint64)
        ent = np.zeros(max(ne.value, 1), np.uint64 if eb.value == 8 else np.uint32)
        lib().ref_get_csr(self.h, C.byref(no), C.byref(ne), C.byref(eb), C.byref(rb), _p(off), _p(ent))
        return off, ent[: ne.value], rb.value, eb.value == 8

    def mutable_lists(self):
        n = self.count()
        lens = np.zeros(n, np.uint64)
        lib().ref_get_mutable(self.h, _p(lens), None)
        flat = np.zeros(max(int(lens.sum()), 1), np.uint32)
        lib().ref_get_mutable(self.h, _p(lens), _p(flat))
        out, pos = [], 0
        for L in lens:
            out.append(flat[pos:pos + int(L)].copy())
            pos += int(L)
        return out
