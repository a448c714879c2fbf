"""hrnn_b200: B200-native HRNN hot path behind the reference's index API.

The Python class :class:`HRNN` mirrors the members of the reference's
``hnswlib::HRNN<float>`` that its drivers call (include/hnswlib/hrnn.h) --
same names, argument meaning and error messages -- and calls the C ABI of
``libhrnn_b200.so`` (declared in include/hrnn_capi.h) through ctypes.  There is
no CPU fallback: importing the package fails if the CUDA library is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhrnn_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"hrnn_b200: CUDA library {LIB_PATH} not built (run `make -C hrnn_b200`)")

_lib = C.CDLL(LIB_PATH)

OK, ERR_ARG, ERR_STATE, ERR_IO, ERR_FORMAT, ERR_CUDA, ERR_NOMEM, ERR_CAPACITY, ERR_LIMIT, ERR_TIMEOUT = range(10)
PREC_FP32_EXACT, PREC_BF16, PREC_INT8 = 0, 1, 2
JOIN_EXACT, JOIN_TENSOR, JOIN_AUDIT = 0, 1, 2

# Every symbol include/hrnn_capi.h declares.
EXPORTS = [
    "hrnn_last_error", "hrnn_version", "hrnn_create", "hrnn_load", "hrnn_save", "hrnn_destroy",
    "hrnn_add_points", "hrnn_refine_knng", "hrnn_build_rknng", "hrnn_build_rknng_mutable",
    "hrnn_search_rknn", "hrnn_search_rknn_batch", "hrnn_search_rknn_batch_device",
    "hrnn_search_plan_create", "hrnn_search_plan_run", "hrnn_search_plan_result", "hrnn_search_plan_run_host",
    "hrnn_search_plan_kernels",
    "hrnn_search_plan_destroy",
    "hrnn_compact_for_serving", "hrnn_insert_dynamic", "hrnn_set_ef", "hrnn_get_info",
    "hrnn_get_search_stats", "hrnn_get_refine_stats", "hrnn_set_precision", "hrnn_set_join_mode", "hrnn_set_autotune", "hrnn_set_l2_order", "hrnn_detect_l2_order", "hrnn_get_knng",
    "hrnn_set_knng", "hrnn_get_rknng", "hrnn_l2_batch", "hrnn_build_rknng_noalloc",
    "hrnn_set_budget", "hrnn_budget_features", "hrnn_budget_train", "hrnn_budget_predict",
    "hrnn_budget_gradients", "hrnn_budget_get_weights", "hrnn_budget_set_weights", "hrnn_get_dynamic_stats",
    "hrnn_dynamic_split", "hrnn_get_kdist", "hrnn_get_rknng_mutable",
]

# Learned-budget MLP: 256 -> 256 -> 256 -> 2; parameters W1 b1 W2 b2 W3 b3 (row-major
# [out, in]), then the input normalisation mean and 1/std.
BUDGET_IN, BUDGET_HIDDEN, BUDGET_OUT = 256, 256, 2
BUDGET_SHAPES = [(256, 256), (256,), (256, 256), (256,), (2, 256), (2,), (256,), (256,)]
BUDGET_PARAMS = sum(int(np.prod(s)) for s in BUDGET_SHAPES)


class Info(C.Structure):
    _fields_ = [
        ("dim", C.c_uint64), ("max_elements", C.c_uint64), ("cur_element_count", C.c_uint64),
        ("M", C.c_uint64), ("maxM", C.c_uint64), ("maxM0", C.c_uint64),
        ("ef_construction", C.c_uint64), ("ef", C.c_uint64), ("K_knng", C.c_uint64),
        ("maxlevel", C.c_int32), ("enterpoint", C.c_uint32),
        ("knng_built", C.c_int32), ("rknng_built", C.c_int32), ("rknng_wide", C.c_int32),
        ("rank_bits", C.c_uint32), ("rknng_entries", C.c_uint64),
        ("serve_mode", C.c_int32), ("max_k_serve", C.c_uint64),
        ("l2_lanes", C.c_int32), ("l2_fused", C.c_int32), ("device_bytes", C.c_uint64),
    ]


class SearchStats(C.Structure):
    _fields_ = [(f, C.c_uint64) for f in (
        "n_queries", "n_dist", "n_expanded", "n_posting", "n_cand", "n_verified", "n_result",
        "n_lowp_decided", "n_fp32_decided", "n_fp64_decided", "n_fp64_flipped", "n_launches")] + [
        ("n_budget", C.c_uint64 * 3),
        ("phase_a_ms", C.c_double), ("phase_b_ms", C.c_double), ("phase_c_ms", C.c_double),
        ("a_warps_per_block", C.c_uint32), ("a_visit_slots", C.c_uint32)]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_}
        d["n_budget"] = list(self.n_budget)
        return d


MAX_ITERS = 64


class RefineStats(C.Structure):
    _fields_ = [("iters", C.c_int32)] + [
        (f, C.c_uint64 * MAX_ITERS) for f in ("join_dists", "updates", "proposals", "sample_entries")] + [
        (f, C.c_double * MAX_ITERS) for f in ("ms", "sample_ms", "join_ms", "bucket_ms", "merge_ms")] + [
        (f, C.c_uint64 * MAX_ITERS) for f in ("screen_survivors", "screen_dense_nodes", "screen_misses")] + [
        ("join_mode", C.c_int32)]

    def as_dict(self):
        k = self.iters
        d = {"iters": k, "join_mode": self.join_mode}
        d.update({f: list(getattr(self, f))[:k] for f, _ in self._fields_[1:-1]})
        return d


class DynamicStats(C.Structure):
    _fields_ = [(f, C.c_uint64) for f in ("n_inserted", "n_batches", "n_dist", "n_proposals", "n_updates")] + [
        (f, C.c_double) for f in ("insert_ms", "rknng_ms", "maintain_ms")]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_vp = C.c_void_p
_sz = C.c_size_t
_lib.hrnn_last_error.restype = C.c_char_p
_lib.hrnn_create.argtypes = [C.POINTER(_vp), _sz, _sz, _sz, _sz, _sz, _sz, C.c_int]
_lib.hrnn_load.argtypes = [C.POINTER(_vp), C.c_char_p, _sz, _sz, C.c_int]
_lib.hrnn_save.argtypes = [_vp, C.c_char_p]
_lib.hrnn_destroy.argtypes = [_vp]
_lib.hrnn_destroy.restype = None
_lib.hrnn_add_points.argtypes = [_vp, _vp, _vp, _sz]
_lib.hrnn_refine_knng.argtypes = [_vp, C.c_int, C.c_int]
_lib.hrnn_build_rknng.argtypes = [_vp]
_lib.hrnn_build_rknng_mutable.argtypes = [_vp]
_lib.hrnn_search_rknn.argtypes = [_vp, _vp, _sz, C.c_float, _sz, _sz, _sz, _vp, _sz, C.POINTER(_sz)]
_lib.hrnn_search_rknn_batch.argtypes = [_vp, _vp, _sz, _vp, _vp, _vp, C.c_float, C.c_uint32, _vp, _vp, _sz]
_lib.hrnn_search_plan_create.argtypes = [_vp, _vp, _sz, _vp, _vp, _vp, C.c_uint32, C.c_uint32, C.c_float,
                                         C.c_uint32, _vp, _vp, _sz, _vp, C.POINTER(_vp)]
_lib.hrnn_search_plan_run.argtypes = [_vp, _vp]
_lib.hrnn_search_plan_result.argtypes = [_vp, _vp, C.POINTER(C.c_uint64), C.POINTER(C.c_int)]
_lib.hrnn_search_plan_kernels.argtypes = [_vp, C.POINTER(_sz)]
_lib.hrnn_search_plan_run_host.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _sz, C.POINTER(C.c_uint64),
                                           C.POINTER(C.c_int), _vp]
_lib.hrnn_search_plan_destroy.argtypes = [_vp]
_lib.hrnn_search_plan_destroy.restype = None
_lib.hrnn_search_rknn_batch_device.argtypes = [_vp, _vp, _sz, _vp, _vp, _vp, C.c_float, C.c_uint32, _vp,
                                               _vp, _sz, C.POINTER(C.c_uint64), _vp]
_lib.hrnn_compact_for_serving.argtypes = [_vp, _sz]
_lib.hrnn_insert_dynamic.argtypes = [_vp, _vp, _vp, _sz, C.c_uint, C.c_int]
_lib.hrnn_set_ef.argtypes = [_vp, _sz]
_lib.hrnn_get_info.argtypes = [_vp, C.POINTER(Info)]
_lib.hrnn_get_search_stats.argtypes = [_vp, C.POINTER(SearchStats)]
_lib.hrnn_get_refine_stats.argtypes = [_vp, C.POINTER(RefineStats)]
_lib.hrnn_get_dynamic_stats.argtypes = [_vp, C.POINTER(DynamicStats)]
_lib.hrnn_set_precision.argtypes = [_vp, C.c_int]
_lib.hrnn_set_join_mode.argtypes = [_vp, C.c_int]
_lib.hrnn_set_autotune.argtypes = [_vp, C.c_int]
_lib.hrnn_set_l2_order.argtypes = [_vp, C.c_int, C.c_int]
_lib.hrnn_detect_l2_order.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int)]
_lib.hrnn_get_knng.argtypes = [_vp, _vp, _vp, _vp]
_lib.hrnn_set_knng.argtypes = [_vp, _vp, _vp, _vp]
_lib.hrnn_get_rknng.argtypes = [_vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint32),
                                C.POINTER(C.c_uint32), _vp, _vp, C.c_int]
_lib.hrnn_l2_batch.argtypes = [_vp, _vp, _sz, _sz, C.c_int, C.c_int, _vp]
_lib.hrnn_set_budget.argtypes = [_vp, C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float]
_lib.hrnn_budget_features.argtypes = [_vp, _vp, _sz, C.c_uint32, C.c_uint32, C.c_uint32, _vp]
_lib.hrnn_budget_train.argtypes = [_vp, _vp, _vp, _sz, C.c_int, C.c_int, C.c_float, C.c_uint64,
                                   C.POINTER(C.c_float)]
_lib.hrnn_budget_predict.argtypes = [_vp, _vp, _sz, _vp]
_lib.hrnn_budget_gradients.argtypes = [_vp, _vp, _vp, _sz, _vp, C.POINTER(C.c_float)]
_lib.hrnn_budget_get_weights.argtypes = [_vp, _vp]
_lib.hrnn_budget_set_weights.argtypes = [_vp, _vp]
_lib.hrnn_build_rknng_noalloc.argtypes = [_vp, _vp, _sz, _sz, _vp, _vp, _sz, C.POINTER(C.c_uint32),
                                          C.POINTER(C.c_int), C.POINTER(C.c_uint64), _vp]


class HrnnError(RuntimeError):
    """std::runtime_error of the reference, carried with the C ABI status code."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


def _check(rc: int):
    if rc != OK:
        raise HrnnError(rc, _lib.hrnn_last_error().decode())


def _p(a: np.ndarray):
    return a.ctypes.data_as(_vp)


def lib():
    return _lib


def detect_l2_order():
    lanes, fused = C.c_int(0), C.c_int(0)
    _check(_lib.hrnn_detect_l2_order(C.byref(lanes), C.byref(fused)))
    return lanes.value, fused.value


def l2_batch(A, B, lanes=16, fused=2) -> np.ndarray:
    """Squared L2 of row pairs on the GPU in the reference's FP32 order."""
    A = np.ascontiguousarray(A, np.float32)
    B = np.ascontiguousarray(B, np.float32)
    out = np.empty(A.shape[0], np.float32)
    _check(_lib.hrnn_l2_batch(_p(A), _p(B), A.shape[0], A.shape[1], lanes, fused, _p(out)))
    return out


def build_rknng_noalloc(d_knn_ids: int, d_knn_cnt: int, n: int, K: int, d_offsets: int, d_entries: int,
                        entries_cap: int, stream: int = 0):
    """Reverse-KNN CSR of a caller-owned device KNN graph, allocating nothing (for
    callers that cannot call cudaMalloc).  Arguments are raw device pointers;
    returns (rank_bits, wide, n_entries).  See include/hrnn_capi.h for the limits."""
    rb, wide, ne = C.c_uint32(0), C.c_int(0), C.c_uint64(0)
    _check(_lib.hrnn_build_rknng_noalloc(_vp(d_knn_ids), _vp(d_knn_cnt), n, K, _vp(d_offsets), _vp(d_entries),
                                         entries_cap, C.byref(rb), C.byref(wide), C.byref(ne), _vp(stream)))
    return rb.value, bool(wide.value), ne.value


def dynamic_split(n: int, seed: int = 42) -> np.ndarray:
    """0..n-1 shuffled by std::shuffle with std::mt19937(seed): the split of the
    reference's src/hrnn_dynamic_test.cpp:200-203 (first split*n build, rest insert)."""
    perm = np.empty(n, np.uint32)
    _check(_lib.hrnn_dynamic_split(C.c_uint64(n), C.c_uint32(seed), _p(perm)))
    return perm


def _split_params(flat):
    out, o = [], 0
    for s in BUDGET_SHAPES:
        k = int(np.prod(s))
        out.append(flat[o:o + k].reshape(s).copy())
        o += k
    return out


def _u32(x, n):
    return np.ascontiguousarray(np.broadcast_to(np.asarray(x, dtype=np.uint32), (n,)))


class HRNN:
    """hnswlib::HRNN<float> with the hot path on the GPU (include/hnswlib/hrnn.h)."""

    def __init__(self, dim: int, max_elements: int = 0, M: int = 16, ef_construction: int = 200,
                 random_seed: int = 100, K_knng: int = 0, device: int = 0, _handle=None):
        self.dim = int(dim)
        self._h = _vp()
        if _handle is not None:
            self._h = _handle
        else:
            _check(_lib.hrnn_create(C.byref(self._h), self.dim, max_elements, M, ef_construction, random_seed,
                                    K_knng, device))

    @classmethod
    def load(cls, path: str, dim: int, max_elements: int = 0, device: int = 0) -> "HRNN":
        """HRNN(space, path, false, max_elements) -- hrnn.h:117."""
        h = _vp()
        _check(_lib.hrnn_load(C.byref(h), path.encode(), dim, max_elements, device))
        return cls(dim, _handle=h)

    def close(self):
        if getattr(self, "_h", None):
            _lib.hrnn_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    # ---- build -------------------------------------------------------------
    def addPoint(self, x, label: int):
        self.add_points(np.asarray(x, np.float32)[None, :], np.asarray([label], np.uint64))

    def add_points(self, X, labels=None):
        X = np.ascontiguousarray(X, np.float32)
        lab = None if labels is None else np.ascontiguousarray(labels, np.uint64)
        _check(_lib.hrnn_add_points(self._h, _p(X), _p(lab) if lab is not None else None, X.shape[0]))

    def refineKNNG(self, num_iters: int = 3, sample_size: int = 20):
        _check(_lib.hrnn_refine_knng(self._h, num_iters, sample_size))

    def buildRKNNG(self):
        _check(_lib.hrnn_build_rknng(self._h))

    def buildRKNNG_mutable(self):
        _check(_lib.hrnn_build_rknng_mutable(self._h))

    def insertPointDynamic(self, X, labels, m_update: int = 0, bidirectional: bool = False):
        X = np.ascontiguousarray(np.atleast_2d(X), np.float32)
        lab = np.ascontiguousarray(np.atleast_1d(labels), np.uint64)
        _check(_lib.hrnn_insert_dynamic(self._h, _p(X), _p(lab), X.shape[0], m_update, int(bidirectional)))

    def saveIndex(self, path: str):
        _check(_lib.hrnn_save(self._h, path.encode()))

    def compactForServing(self, max_k_serve: int):
        _check(_lib.hrnn_compact_for_serving(self._h, max_k_serve))

    def setEf(self, ef: int):
        _check(_lib.hrnn_set_ef(self._h, ef))

    def set_l2_order(self, lanes: int, fused: int):
        _check(_lib.hrnn_set_l2_order(self._h, lanes, fused))

    def set_precision(self, precision: int):
        """PREC_FP32_EXACT (bit-identical to the reference), PREC_BF16 or PREC_INT8."""
        _check(_lib.hrnn_set_precision(self._h, precision))

    def set_autotune(self, enable: bool):
        """Time the beam-search launch shapes on the first large batch (default on)."""
        _check(_lib.hrnn_set_autotune(self._h, 1 if enable else 0))

    def set_join_mode(self, mode: int):
        """Local join of refineKNNG: JOIN_EXACT (the default), JOIN_TENSOR (BF16
        tensor-core screen, exact FP32 for the pairs it keeps; same lists), or
        JOIN_AUDIT (screen decisions checked against every pair's exact distance)."""
        _check(_lib.hrnn_set_join_mode(self._h, mode))

    # ---- search ------------------------------------------------------------
    def searchRknn(self, q, m: int, threshold: float, k: int, K_prime: int, ef_search: int) -> list:
        """searchRknn -- hrnn.h:1966; labels in ascending internal-id order."""
        return [int(x) for x in self.search_rknn_batch(np.asarray(q, np.float32)[None, :], m, K_prime,
                                                       ef_search, threshold, k)[0]]

    def search_rknn_batch(self, Q, m, K_prime, ef_search, threshold: float = 1.0, k: int = 10):
        """Batch of searchRknn with host arrays; returns one label array per query."""
        Q = np.ascontiguousarray(Q, np.float32)
        nq = Q.shape[0]
        mm, kp, ef = _u32(m, nq), _u32(K_prime, nq), _u32(ef_search, nq)
        off, lab = self.search_rknn_batch_csr(Q, mm, kp, ef, threshold, k)
        return [lab[off[i]:off[i + 1]] for i in range(nq)]

    def search_rknn_batch_csr(self, Q, m, K_prime, ef_search, threshold: float = 1.0, k: int = 10):
        """Batch of searchRknn with host arrays; returns (offsets[nq + 1], labels):
        query i's labels are labels[offsets[i]:offsets[i + 1]], ascending internal id."""
        Q = np.ascontiguousarray(Q, np.float32)
        nq = Q.shape[0]
        mm, kp, ef = _u32(m, nq), _u32(K_prime, nq), _u32(ef_search, nq)
        off = np.empty(nq + 1, np.uint64)
        cap = max(16, int(np.sum(mm.astype(np.int64)) * 64))
        lab = np.empty(cap, np.uint64)
        rc = _lib.hrnn_search_rknn_batch(self._h, _p(Q), nq, _p(mm), _p(kp), _p(ef), threshold, k, _p(off),
                                         _p(lab), cap)
        if rc == ERR_CAPACITY:
            cap = int(off[-1])
            lab = np.empty(max(cap, 1), np.uint64)
            rc = _lib.hrnn_search_rknn_batch(self._h, _p(Q), nq, _p(mm), _p(kp), _p(ef), threshold, k,
                                             _p(off), _p(lab), cap)
        _check(rc)
        return off, lab[:int(off[-1])]

    def search_rknn_batch_host(self, q_ptr, nq, m_ptr, kp_ptr, ef_ptr, threshold, k, off_ptr, lab_ptr, cap) -> int:
        """hrnn_search_rknn_batch on raw HOST pointers (e.g. pinned buffers): copies
        in, searches, copies out and waits; returns the total result count."""
        _check(_lib.hrnn_search_rknn_batch(self._h, _vp(q_ptr), nq, _vp(m_ptr), _vp(kp_ptr), _vp(ef_ptr), threshold,
                                           k, _vp(off_ptr), _vp(lab_ptr), cap))
        return int(C.c_uint64.from_address(off_ptr + 8 * nq).value)

    def search_rknn_batch_device(self, q_ptr, nq, m_ptr, kp_ptr, ef_ptr, threshold, k, off_ptr, lab_ptr,
                                 cap, stream=0):
        """Device-pointer batch (ints are raw CUDA pointers); returns the total result count."""
        tot = C.c_uint64(0)
        _check(_lib.hrnn_search_rknn_batch_device(self._h, _vp(q_ptr), nq, _vp(m_ptr), _vp(kp_ptr), _vp(ef_ptr),
                                                  threshold, k, _vp(off_ptr), _vp(lab_ptr), cap, C.byref(tot),
                                                  _vp(stream)))
        return tot.value

    def search_plan(self, q_ptr, nq, m_ptr, kp_ptr, ef_ptr, m_max, ef_max, threshold, k, off_ptr, lab_ptr, cap,
                    stream=0) -> "SearchPlan":
        """A captured search plan over fixed device buffers (ints are raw CUDA
        pointers): run() replays the whole batch search as one CUDA graph."""
        out = _vp()
        _check(_lib.hrnn_search_plan_create(self._h, _vp(q_ptr), nq, _vp(m_ptr), _vp(kp_ptr), _vp(ef_ptr), m_max,
                                            ef_max, threshold, k, _vp(off_ptr), _vp(lab_ptr), cap, _vp(stream),
                                            C.byref(out)))
        return SearchPlan(self, out)

    # ---- learned search budget (no counterpart in the reference) -------------
    def set_budget(self, enable: bool, m0: int = 1, m1: int = 3, ef: int = 0, confidence: float = 0.9):
        """Serve searches with the learned budget when enabled: levels of m0 / m1
        proxies; ef = 0 takes them from the caller's beam, ef > 0 from a beam of ef
        (with a second search for the other queries)."""
        _check(_lib.hrnn_set_budget(self._h, int(enable), m0, m1, ef, confidence))

    def budget_features(self, Q, k: int, m: int = 1, ef_search: int = 1) -> np.ndarray:
        """The MLP's 256 features of each query, from the frontier of a search with
        (m, ef_search) -- the budget's (m1, ef) in two-pass mode."""
        Q = np.ascontiguousarray(Q, np.float32)
        f = np.zeros((Q.shape[0], BUDGET_IN), np.float32)
        _check(_lib.hrnn_budget_features(self._h, _p(Q), Q.shape[0], k, m, ef_search, _p(f)))
        return f

    def budget_train(self, feat, labels, epochs: int = 10, batch: int = 1024, lr: float = 1e-3,
                     seed: int = 0) -> float:
        feat = np.ascontiguousarray(feat, np.float32)
        labels = np.ascontiguousarray(labels, np.uint8)
        assert feat.shape[1:] == (BUDGET_IN,) and labels.shape == (feat.shape[0], BUDGET_OUT)
        loss = C.c_float(0)
        _check(_lib.hrnn_budget_train(self._h, _p(feat), _p(labels), feat.shape[0], epochs, batch, lr, seed,
                                      C.byref(loss)))
        return loss.value

    def budget_predict(self, feat) -> np.ndarray:
        feat = np.ascontiguousarray(feat, np.float32)
        z = np.zeros((feat.shape[0], BUDGET_OUT), np.float32)
        _check(_lib.hrnn_budget_predict(self._h, _p(feat), feat.shape[0], _p(z)))
        return z

    def budget_gradients(self, feat, labels):
        """Gradients of the mean BCE for W1 b1 W2 b2 W3 b3 and the loss."""
        feat = np.ascontiguousarray(feat, np.float32)
        labels = np.ascontiguousarray(labels, np.uint8)
        g = np.zeros(BUDGET_PARAMS, np.float32)
        loss = C.c_float(0)
        _check(_lib.hrnn_budget_gradients(self._h, _p(feat), _p(labels), feat.shape[0], _p(g), C.byref(loss)))
        return _split_params(g)[:6], loss.value

    def budget_get_weights(self):
        g = np.zeros(BUDGET_PARAMS, np.float32)
        _check(_lib.hrnn_budget_get_weights(self._h, _p(g)))
        return _split_params(g)

    def budget_set_weights(self, params):
        flat = np.concatenate([np.asarray(p, np.float32).ravel() for p in params])
        assert flat.size == BUDGET_PARAMS
        _check(_lib.hrnn_budget_set_weights(self._h, _p(flat)))

    # ---- inspection ----------------------------------------------------------
    def info(self) -> dict:
        i = Info()
        _check(_lib.hrnn_get_info(self._h, C.byref(i)))
        return {f: getattr(i, f) for f, _ in Info._fields_}

    def last_search_stats(self) -> dict:
        s = SearchStats()
        _check(_lib.hrnn_get_search_stats(self._h, C.byref(s)))
        return s.as_dict()

    def last_dynamic_stats(self) -> dict:
        s = DynamicStats()
        _check(_lib.hrnn_get_dynamic_stats(self._h, C.byref(s)))
        return s.as_dict()

    def last_refine_stats(self) -> dict:
        s = RefineStats()
        _check(_lib.hrnn_get_refine_stats(self._h, C.byref(s)))
        return s.as_dict()

    def getCurrentElementCount(self) -> int:
        return self.info()["cur_element_count"]

    @property
    def K_knng_(self) -> int:
        return self.info()["K_knng"]

    @property
    def knng_built_(self) -> bool:
        return bool(self.info()["knng_built"])

    @property
    def rknng_built_(self) -> bool:
        return bool(self.info()["rknng_built"])

    def get_knng(self):
        inf = self.info()
        n, K = inf["cur_element_count"], inf["K_knng"]
        ids = np.zeros((n, K), np.uint32)
        d = np.zeros((n, K), np.float32)
        cnt = np.zeros(n, np.uint32)
        _check(_lib.hrnn_get_knng(self._h, _p(ids), _p(d), _p(cnt)))
        return ids, d, cnt

    def get_rknng_mutable(self):
        """The mutable reverse lists (rknng_lists_ of hrnn.h:1942-1959) as one owner
        array per element, in the device's order."""
        n = self.getCurrentElementCount()
        lens = np.zeros(n, np.uint64)
        _check(_lib.hrnn_get_rknng_mutable(self._h, _p(lens), None))
        flat = np.zeros(max(int(lens.sum()), 1), np.uint32)
        _check(_lib.hrnn_get_rknng_mutable(self._h, _p(lens), _p(flat)))
        off = np.zeros(n + 1, np.int64)
        off[1:] = np.cumsum(lens.astype(np.int64))
        return [flat[off[i]:off[i + 1]] for i in range(n)]

    def get_kdist(self, k: int) -> np.ndarray:
        """kdist(p, k-1) of every element (FLT_MAX where the list is shorter than
        k): the radius the verification compares against (hrnn.h:286-293)."""
        out = np.empty(self.getCurrentElementCount(), np.float32)
        _check(_lib.hrnn_get_kdist(self._h, C.c_uint32(k), _p(out)))
        return out

    def get_knng_column(self, j: int):
        """(ids[:, j], dists[:, j], cnt) of the KNN slot: e.g. j = k - 1 gives the
        k-th neighbour distance the verification compares against (hrnn.h:286-293;
        meaningful where cnt > j)."""
        ids, d, cnt = self.get_knng()
        return ids[:, j].copy(), d[:, j].copy(), cnt

    def set_knng(self, ids, dists, cnt):
        ids = np.ascontiguousarray(ids, np.uint32)
        dists = np.ascontiguousarray(dists, np.float32)
        cnt = np.ascontiguousarray(cnt, np.uint32)
        _check(_lib.hrnn_set_knng(self._h, _p(ids), _p(dists), _p(cnt)))

    def get_rknng(self, reference_order: bool = False):
        no, ne = C.c_uint64(0), C.c_uint64(0)
        eb, rb = C.c_uint32(0), C.c_uint32(0)
        _check(_lib.hrnn_get_rknng(self._h, C.byref(no), C.byref(ne), C.byref(eb), C.byref(rb), None, None, 0))
        off = np.zeros(no.value, np.uint64)
        ent = np.zeros(max(ne.value, 1), np.uint64 if eb.value == 8 else np.uint32)
        _check(_lib.hrnn_get_rknng(self._h, C.byref(no), C.byref(ne), C.byref(eb), C.byref(rb), _p(off), _p(ent),
                                   int(reference_order)))
        return off, ent[: ne.value], rb.value, eb.value == 8


class SearchPlan:
    """hrnn_search_plan_*: the batch search recorded once as a CUDA graph."""

    def __init__(self, index, handle):
        self._index = index  # keeps the index alive while the plan exists
        self._p = handle

    def run(self, stream=0):
        _check(_lib.hrnn_search_plan_run(self._p, _vp(stream)))

    def result(self, stream=0):
        """Waits for the stream; returns (total results, clamped flag)."""
        tot, cl = C.c_uint64(0), C.c_int(0)
        _check(_lib.hrnn_search_plan_result(self._p, _vp(stream), C.byref(tot), C.byref(cl)))
        return tot.value, bool(cl.value)

    def run_host(self, q_ptr, m_ptr, kp_ptr, ef_ptr, off_ptr, lab_ptr, cap, stream=0):
        """One run on a host batch (ints are raw host pointers): copies in, replays,
        waits, copies the offsets and labels out; returns (total, clamped)."""
        tot, cl = C.c_uint64(0), C.c_int(0)
        _check(_lib.hrnn_search_plan_run_host(self._p, _vp(q_ptr), _vp(m_ptr), _vp(kp_ptr), _vp(ef_ptr),
                                              _vp(off_ptr), _vp(lab_ptr), cap, C.byref(tot), C.byref(cl),
                                              _vp(stream)))
        return tot.value, bool(cl.value)

    def kernels(self) -> int:
        """Kernel launches one run makes (the graph's kernel nodes)."""
        n = C.c_size_t(0)
        _check(_lib.hrnn_search_plan_kernels(self._p, C.byref(n)))
        return n.value

    def close(self):
        if self._p:
            _lib.hrnn_search_plan_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
