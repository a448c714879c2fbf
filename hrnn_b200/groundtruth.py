"""Reverse-kNN ground truth on the GPU, every membership decided in float64.

RkNN(q, k) = { x : dist(q, x) <= dist(x, x_k) }, x_k the k-th nearest other
point of x -- the definition and the file layout of the reference's
scripts/gen_rknn_gt.py (:5-8, :10-14):

    [nq: u32][offsets: (nq+1) u32][ids: total u32][dists: total f32]

with each query's ids ordered by distance.  The reference takes the squared
distances in float32; here float32 GEMMs only screen (with a margin that bounds
their rounding error) and every kept distance and every comparison is made in
float64, so the ground truth does not depend on float32 rounding.

    python -m hrnn_b200.groundtruth --base base.fbin --query query.fbin --k 10 \\
        --output rknn_gt.bin [--chunk_base 2048] [--chunk_query 256]

(the flags of scripts/gen_rknn_gt.py; torch with CUDA is the only dependency).
"""
from __future__ import annotations

import argparse
import time

import numpy as np


def read_fbin(path: str) -> np.ndarray:
    """fbin layout [n: u32][d: u32][n*d f32] (include/utils.h:32-47)."""
    with open(path, "rb") as f:
        n, d = np.fromfile(f, dtype=np.uint32, count=2)
        return np.fromfile(f, dtype=np.float32, count=int(n) * int(d)).reshape(int(n), int(d))


def write_fbin(path: str, X: np.ndarray) -> None:
    with open(path, "wb") as f:
        np.array(X.shape, dtype=np.uint32).tofile(f)
        np.ascontiguousarray(X, dtype=np.float32).tofile(f)


def _margin(na, nb):
    # bound on the float32 GEMM error of ||a||^2 - 2 a.b + ||b||^2 (relative 1e-4
    # of the norms is far above the accumulated rounding for d <= 4096)
    return 1e-4 * (na + nb) + 1e-3


def kth_radius_fp64(X: np.ndarray, k: int, device=None, chunk: int = 2048, rows=None) -> np.ndarray:
    """Float64 squared distance of every point (or of the points `rows`) to its
    k-th nearest other point."""
    import torch
    device = device or torch.device("cuda", torch.cuda.current_device())
    torch.backends.cuda.matmul.allow_tf32 = False
    n = X.shape[0]
    if n <= k:
        raise ValueError("kth_radius_fp64: need more than k points")
    Xt = torch.from_numpy(np.ascontiguousarray(X, np.float32)).to(device)
    X64 = Xt.double()
    nx64 = (X64 ** 2).sum(1)
    nx = nx64.float()
    nxmax = nx64.max()
    R = torch.arange(n, device=device) if rows is None else torch.from_numpy(np.asarray(rows, np.int64)).to(device)
    chunk = max(1, min(chunk, (1 << 31) // n))  # a chunk's float32 distance rows stay within 8 GB
    out = torch.empty(len(R), dtype=torch.float64, device=device)
    pad = min(n - 1, k + 16)
    exact_rows = []
    for s in range(0, len(R), chunk):
        e = min(len(R), s + chunk)
        r = R[s:e]
        D = nx[r, None] - 2.0 * (Xt[r] @ Xt.T) + nx[None, :]
        D[torch.arange(e - s, device=device), r] = float("inf")
        vals, idx = torch.topk(D, pad, dim=1, largest=False, sorted=True)
        ex = ((X64[r, None, :] - X64[idx]) ** 2).sum(2)
        kth = torch.sort(ex, dim=1).values[:, k - 1]
        out[s:e] = kth
        # every point outside the pad candidates has a float32 distance >= the last
        # candidate's: if that minus the margin still exceeds kth, kth is exact
        ok = (vals[:, -1].double() - _margin(nx64[r], nxmax)) > kth
        if not bool(ok.all()):
            exact_rows.extend((torch.nonzero(~ok).flatten() + s).tolist())
    for j in exact_rows:  # the whole row in float64
        i = int(R[j])
        d = ((X64 - X64[i]) ** 2).sum(1)
        d[i] = float("inf")
        out[j] = torch.kthvalue(d, k).values
    return out.cpu().numpy()


def rknn_fp64_bounded(X: np.ndarray, Q: np.ndarray, kth_upper: np.ndarray, k: int, device=None,
                      q_chunk: int = 64, x_chunk: int = 1 << 21):
    """RkNN ground truth of a query subset without every point's k-th radius:
    kth_upper[x] >= x's true k-th radius (e.g. the k-th distance of an approximate
    KNN list -- the k-th smallest of any k other points' distances is at least
    the true one) screens the points, the exact float64 radius is computed only
    for the points some query may reach, and every decision is float64.
    Returns what rknn_fp64 returns, and the number of radii computed."""
    import torch
    device = device or torch.device("cuda", torch.cuda.current_device())
    torch.backends.cuda.matmul.allow_tf32 = False
    n = X.shape[0]
    Xt = torch.from_numpy(np.ascontiguousarray(X, np.float32)).to(device)
    nx64 = (Xt.double() ** 2).sum(1)
    up = torch.from_numpy(np.asarray(kth_upper, np.float64)).to(device)
    cand = []
    for s in range(0, Q.shape[0], q_chunk):
        q = torch.from_numpy(np.ascontiguousarray(Q[s:s + q_chunk], np.float32)).to(device)
        nq = (q.double() ** 2).sum(1)
        for x0 in range(0, n, x_chunk):
            x1 = min(n, x0 + x_chunk)
            D = nq[:, None] - 2.0 * (q @ Xt[x0:x1].T).double() + nx64[None, x0:x1]
            hit = torch.nonzero(D <= up[None, x0:x1] + _margin(nq[:, None], nx64[None, x0:x1]))
            if len(hit):
                cand.append(hit[:, 1] + x0)
            del D
    rows = torch.unique(torch.cat(cand)).cpu().numpy() if cand else np.zeros(0, np.int64)
    kth = np.full(n, -1.0)  # radius unknown = unreachable: -1 admits nothing
    if len(rows):
        kth[rows] = kth_radius_fp64(X, k, device, rows=rows)
    return rknn_fp64(X, Q, kth, device, chunk=q_chunk), int(len(rows))


def rknn_fp64(X: np.ndarray, Q: np.ndarray, kth: np.ndarray, device=None, chunk: int = 256):
    """Per query: (ids ascending by distance, float64 squared distances)."""
    import torch
    device = device or torch.device("cuda", torch.cuda.current_device())
    torch.backends.cuda.matmul.allow_tf32 = False
    Xt = torch.from_numpy(np.ascontiguousarray(X, np.float32)).to(device)
    X64 = Xt.double()
    nx = (X64 ** 2).sum(1)
    kt = torch.from_numpy(np.asarray(kth, np.float64)).to(device)
    out = []
    for s in range(0, Q.shape[0], chunk):
        q = torch.from_numpy(np.ascontiguousarray(Q[s:s + chunk], np.float32)).to(device)
        q64 = q.double()
        nq = (q64 ** 2).sum(1)
        D = nq[:, None] - 2.0 * (q @ Xt.T).double() + nx[None, :]
        cand = torch.nonzero(D <= kt[None, :] + _margin(nq[:, None], nx[None, :]))
        qi, xi = cand[:, 0], cand[:, 1]
        ex = ((q64[qi] - X64[xi]) ** 2).sum(1)
        keep = ex <= kt[xi]
        qi, xi, ex = qi[keep].cpu().numpy(), xi[keep].cpu().numpy(), ex[keep].cpu().numpy()
        for j in range(q.shape[0]):
            sel = qi == j
            ids, ds = xi[sel], ex[sel]
            o = np.lexsort((ids, ds))
            out.append((ids[o].astype(np.uint32), ds[o]))
    return out


def write_rknn_gt(path: str, gt) -> None:
    """gt: per query (ids, distances) as rknn_fp64 returns them."""
    off = np.zeros(len(gt) + 1, np.uint32)
    for i, (ids, _) in enumerate(gt):
        off[i + 1] = off[i] + len(ids)
    with open(path, "wb") as f:
        np.array([len(gt)], np.uint32).tofile(f)
        off.tofile(f)
        for ids, _ in gt:
            np.asarray(ids, np.uint32).tofile(f)
        for _, ds in gt:
            np.asarray(ds, np.float32).tofile(f)


def read_rknn_gt(path: str):
    with open(path, "rb") as f:
        nq = int(np.fromfile(f, np.uint32, 1)[0])
        off = np.fromfile(f, np.uint32, nq + 1)
        ids = np.fromfile(f, np.uint32, int(off[-1]))
        ds = np.fromfile(f, np.float32, int(off[-1]))
    return [(ids[off[i]:off[i + 1]], ds[off[i]:off[i + 1]]) for i in range(nq)]


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="RkNN ground truth, float64 decisions on the GPU")
    ap.add_argument("--base", required=True)
    ap.add_argument("--query", required=True)
    ap.add_argument("--k", type=int, default=10)
    ap.add_argument("--output", required=True)
    ap.add_argument("--chunk_base", type=int, default=2048)
    ap.add_argument("--chunk_query", type=int, default=256)
    a = ap.parse_args(argv)
    X, Q = read_fbin(a.base), read_fbin(a.query)
    print(f"  base n={X.shape[0]} d={X.shape[1]}, queries nq={Q.shape[0]}, k={a.k}")
    t0 = time.time()
    kth = kth_radius_fp64(X, a.k, chunk=a.chunk_base)
    t1 = time.time()
    gt = rknn_fp64(X, Q, kth, chunk=a.chunk_query)
    write_rknn_gt(a.output, gt)
    sizes = np.array([len(i) for i, _ in gt])
    print(f"  k-th radii {t1 - t0:.1f}s, RkNN {time.time() - t1:.1f}s; mean |RkNN| {sizes.mean():.2f}, "
          f"empty {(sizes == 0).sum()}; wrote {a.output}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
