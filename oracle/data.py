"""Seeded synthetic inputs and FP64 ground truth (test / measurement infrastructure).

The reference's datasets (SIFT, GIST, MSMARCO, Msong) are not available; seeded
Gaussian mixtures with the benchmark's shapes stand in for them:
centres ~ N(0, 4 I) drawn with default_rng(centre_seed), equal or Dirichlet(1)
weights, points = centre[label] + N(0, sigma^2 I), float32.

The RkNN ground truth follows the definition in scripts/gen_rknn_gt.py:5-8:
RkNN(q) = { x : dist(x, q) <= dist(x, x_k) }, x_k the k-th nearest neighbour of
x among the other points, with every distance evaluated in float64.
"""
from __future__ import annotations

import numpy as np


def mixture(n: int, d: int, C: int, sigma: float, centre_seed: int, draw_seed: int,
            dirichlet: bool = False) -> np.ndarray:
    rc = np.random.default_rng(centre_seed)
    centres = rc.normal(0.0, 2.0, (C, d))
    w = rc.dirichlet(np.ones(C)) if dirichlet else np.full(C, 1.0 / C)
    r = np.random.default_rng(draw_seed)
    lab = r.choice(C, size=n, p=w)
    return (centres[lab] + r.normal(0.0, sigma, (n, d))).astype(np.float32)


def write_fbin(path: str, X: np.ndarray) -> None:
    """fbin layout [n:u32][d:u32][n*d f32] (include/utils.h:32-47)."""
    with open(path, "wb") as f:
        np.array(X.shape, dtype=np.uint32).tofile(f)
        np.ascontiguousarray(X, dtype=np.float32).tofile(f)


def read_fbin(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        n, d = np.fromfile(f, dtype=np.uint32, count=2)
        return np.fromfile(f, dtype=np.float32, count=int(n) * int(d)).reshape(int(n), int(d))


def kth_nn_fp64(X: np.ndarray, k: int, block: int = 2048) -> np.ndarray:
    """Exact float64 squared distance to the k-th nearest other point."""
    Xd = X.astype(np.float64)
    nx = (Xd * Xd).sum(1)
    out = np.empty(len(X))
    pad = min(len(X) - 1, k + 8)
    for s in range(0, len(X), block):
        e = min(len(X), s + block)
        D = nx[s:e, None] - 2.0 * Xd[s:e] @ Xd.T + nx[None, :]
        D[np.arange(e - s), np.arange(s, e)] = np.inf
        part = np.argpartition(D, pad, axis=1)[:, : pad + 1]
        diff = Xd[s:e, None, :] - Xd[part]
        ex = (diff * diff).sum(2)
        ex[part == np.arange(s, e)[:, None]] = np.inf
        ex.sort(axis=1)
        out[s:e] = ex[:, k - 1]
    return out


def rknn_gt_fp64(X: np.ndarray, Q: np.ndarray, kth: np.ndarray):
    """Per-query sorted id arrays of { x : ||q-x||^2 <= kth[x] } in float64."""
    Xd = X.astype(np.float64)
    res = []
    for q in Q.astype(np.float64):
        dq = ((Xd - q) ** 2).sum(1)
        res.append(np.nonzero(dq <= kth)[0].astype(np.uint32))
    return res


def write_rknn_gt(path: str, X: np.ndarray, Q: np.ndarray, gt) -> None:
    """scripts/gen_rknn_gt.py:10-14 layout: [nq][offsets (nq+1) u32][ids u32][dists f32],
    each query's ids ordered by distance."""
    Xd = X.astype(np.float64)
    off = [0]
    ids, ds = [], []
    for qi, g in enumerate(gt):
        dq = ((Xd[g] - Q[qi].astype(np.float64)) ** 2).sum(1)
        o = np.argsort(dq, kind="stable")
        ids.append(g[o])
        ds.append(dq[o].astype(np.float32))
        off.append(off[-1] + len(g))
    with open(path, "wb") as f:
        np.array([len(gt)], np.uint32).tofile(f)
        np.array(off, np.uint32).tofile(f)
        (np.concatenate(ids) if ids else np.zeros(0, np.uint32)).astype(np.uint32).tofile(f)
        (np.concatenate(ds) if ds else np.zeros(0, np.float32)).astype(np.float32).tofile(f)


def macro_recall(gt, results) -> float:
    """Average over queries with non-empty GT of |res ∩ gt| / |gt| (include/utils.h:135-157)."""
    s, c = 0.0, 0
    for g, r in zip(gt, results):
        if len(g) == 0:
            continue
        s += len(np.intersect1d(g, np.asarray(r, dtype=np.uint32))) / len(g)
        c += 1
    return s / c if c else 0.0
