"""The multi-GPU form of the bench is replicas: each rank answers its own query
stream and the job reports the slowest rank's time.  Two gloo ranks on the CPU
check that reduction and that the replicas' query streams differ."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        W = dict(bench.WORKLOADS["plain-100k-d128-K100"], nq=16)
        q = bench.replica_queries(W, rank)
        slow = bench.max_over_ranks(torch, 10.0 + 5.0 * rank, torch.device("cpu"), world)
        # everyone sees every replica's first query through a gather
        t = torch.from_numpy(q[:1].copy())
        gathered = [torch.zeros_like(t) for _ in range(world)]
        dist.all_gather(gathered, t)
        out[rank] = (slow, [g.numpy() for g in gathered])
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replicas_two_gloo_ranks():
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        res = dict(out)
    assert res[0][0] == res[1][0] == 15.0
    g0, g1 = res[0][1]
    assert not np.array_equal(g0, g1)  # distinct query streams
    assert np.array_equal(res[1][1][0], g0)
