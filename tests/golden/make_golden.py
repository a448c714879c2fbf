"""Generates the committed golden fixtures from the REFERENCE itself.

Run in a container where the reference tree is present and oracle/_ref is built
(`make -C oracle`).  Every expected value below is an output of the reference's
own code (include/hnswlib/hrnn.h compiled from its sources), on seeded inputs:

  small_index.idx.gz   hrnn_build flow on 1500 x 32 points (M=8, ef_c=64, K=24,
                       nn_iters=3, nn_sample=12, one thread), saved by saveIndex
  small_pre_refine.npz the KNN graph before refineKNNG and the one after it
  small_search.npz     queries and searchRknn answers for a parameter sweep
  l2_pairs.npz         L2Space distances for several dims (16-lane AVX-512 build)

    python tests/golden/make_golden.py
"""
import gzip
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import data, ref  # noqa: E402

N, D, M, EFC, K, ITERS, S = 1500, 32, 8, 64, 24, 3, 12
SWEEP = [  # (m, K', ef, threshold, k)
    (1, 24, 16, 1.0, 5), (3, 24, 32, 1.0, 5), (5, 12, 40, 1.0, 5), (10, 24, 40, 1.0, 10),
    (20, 8, 64, 1.0, 3), (5, 24, 8, 2.0, 5), (10, 24, 40, 3.0, 5), (1, 1, 1, 1.0, 1),
    (8, 100, 20, 1.0, 30), (0, 24, 16, 1.0, 5), (4, 0, 16, 1.0, 5), (12, 24, 12, 1.0, 24),
]


def main():
    X = data.mixture(N, D, 12, 1.0, 11, 11)
    Q = data.mixture(120, D, 12, 1.0, 11, 12)
    r = ref.RefIndex.create(D, N, M, EFC, 100, K)
    r.add_points(X, threads=1)
    pre = r.knng(K)
    r.refine(ITERS, S, threads=1)
    post = r.knng(K)
    r.build_rknng()
    tmp = os.path.join(HERE, "_small.idx")
    r.save(tmp)
    with open(tmp, "rb") as f, gzip.open(os.path.join(HERE, "small_index.idx.gz"), "wb", 9) as g:
        g.write(f.read())
    os.remove(tmp)
    np.savez_compressed(os.path.join(HERE, "small_pre_refine.npz"), X=X, pre_ids=pre[0], pre_dists=pre[1],
                        pre_cnt=pre[2], post_ids=post[0], post_dists=post[1], post_cnt=post[2],
                        iters=ITERS, sample=S)
    out = {"Q": Q, "sweep": np.array(SWEEP, dtype=np.float64)}
    for i, (m, kp, ef, th, k) in enumerate(SWEEP):
        res = r.search_batch(Q, int(m), int(kp), int(ef), threshold=th, k=int(k))
        out[f"off_{i}"] = np.cumsum([0] + [len(x) for x in res]).astype(np.uint64)
        out[f"lab_{i}"] = np.concatenate(res).astype(np.uint64) if res else np.zeros(0, np.uint64)
    np.savez_compressed(os.path.join(HERE, "small_search.npz"), **out)
    rng = np.random.default_rng(5)
    l2 = {}
    for d in (7, 16, 20, 32, 36, 96, 128, 256):
        A = rng.normal(0, 2, (96, d)).astype(np.float32)
        B = rng.normal(0, 2, (96, d)).astype(np.float32)
        l2[f"A_{d}"], l2[f"B_{d}"], l2[f"D_{d}"] = A, B, ref.l2_batch(A, B)
    np.savez_compressed(os.path.join(HERE, "l2_pairs.npz"), **l2)
    print("golden fixtures written")


if __name__ == "__main__":
    main()
