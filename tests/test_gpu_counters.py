"""Work counters of the GPU search against the oracle's on the same index: the
number of expanded nodes is identical (same expansion order); distance
evaluations may exceed the oracle's only through visited-cache misses."""
import numpy as np
import pytest

from oracle import data, idx, port

import hrnn_b200 as H

pytestmark = pytest.mark.gpu


def test_work_counters_vs_oracle(golden_idx):
    f = idx.read_idx(golden_idx)
    O = port.OracleIndex(f)
    h = H.HRNN.load(golden_idx, 32)
    Q = data.mixture(200, 32, 12, 1.0, 11, 55)
    h.search_rknn_batch(Q, 10, 24, 64, k=10)
    g = h.last_search_stats()
    tot = {"n_dist": 0, "n_expanded": 0, "n_posting": 0, "n_result": 0}
    for q in Q:
        _, _, st = O.search_one(q, 10, 24, 64, k=10)
        for k in tot:
            tot[k] += st[k]
    assert g["n_expanded"] == tot["n_expanded"]
    assert g["n_posting"] == tot["n_posting"] and g["n_result"] == tot["n_result"]
    assert tot["n_dist"] <= g["n_dist"] <= 1.5 * tot["n_dist"]
    print("gpu n_dist", g["n_dist"], "oracle", tot["n_dist"])
