#!/usr/bin/env python3
"""Benchmark of the B200 HRNN hot path: RkNN queries/s at macro recall >= 0.95 (k=10)
and the KNN-graph build time, on the 1M x 128, K_knng=500 Gaussian-mixture index.

One step = one batch of queries (10,000 by default) answered by the batched
search on an index resident in HBM.  `value` is whole-job queries/s over the
timed steps (CUDA events on the launching stream, max over ranks); `e2e` is
the same metric through the public host-buffer entry point
(hrnn_search_rknn_batch: queries copied in, labels copied out inside the call).
The index (GPU HNSW insertion + NNDescent + reverse CSR) is built first; its
build times are reported under "knng_build".

Multi-GPU: search does not shard (every query needs the whole index), so N ranks
run N independent replicas, each answering its own query batch ("replicas only").

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
                  [--workload mixed-1M-d128-K500 | plain-100k-d128-K100]

--impl reference times the reference's own searchRknn (oracle/_ref: include/
hnswlib/hrnn.h compiled from its sources) with all host threads, on the same
index file, workload, metric and parameters; rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # The configuration the metric is quoted on: 1M x 128, Dirichlet(1) mixture of
    # 256 Gaussians (centres ~ N(0, 4I), sigma 1, seed 2), K_knng=500.
    "mixed-1M-d128-K500": dict(n=1_000_000, d=128, C=256, sigma=1.0, seed=2, dirichlet=True, nq=10_000,
                               qseed=1002, M=16, efc=400, K=500, iters=10, S=50, k=10, Kp=500, ef=200,
                               m_sweep=[1, 2, 3, 4, 5, 6, 8, 10, 20, 50]),
    # Profiling case: the same mixture at half the size (vectors 256 MB > L2), K_knng=250.
    "mixed-500k-d128-K250": dict(n=500_000, d=128, C=256, sigma=1.0, seed=2, dirichlet=True, nq=2_000,
                                 qseed=1002, M=16, efc=400, K=250, iters=10, S=50, k=10, Kp=250, ef=200,
                                 m_sweep=[1, 2, 3, 4, 5, 6, 8, 10, 20, 50]),
    # Build profiling case: the 1M mixture's generator at 200k points, K_knng=500,
    # two NNDescent iterations (used with --build-only).
    "build-200k-d128-K500": dict(n=200_000, d=128, C=256, sigma=1.0, seed=2, dirichlet=True, nq=1_000,
                                 qseed=1002, M=16, efc=400, K=500, iters=2, S=50, k=10, Kp=500, ef=200,
                                 m_sweep=[5]),
    # Join profiling case: 50k points of the same generator, K_knng=100, three
    # NNDescent iterations (about 2 GB on the device; used with --build-only).
    "build-50k-d128-K100": dict(n=50_000, d=128, C=256, sigma=1.0, seed=2, dirichlet=True, nq=1_000,
                                qseed=1002, M=16, efc=100, K=100, iters=3, S=50, k=10, Kp=100, ef=200,
                                m_sweep=[5]),
    # Large single-GPU case: 10M x 96, 1024 equal Gaussians (sigma 1, seed 4),
    # K_knng=200 (8 GB of ids + 8 GB of distances), reverse CSR of 2e9 entries;
    # 100,000 queries per step, recall against a float64 ground truth of the first
    # 5,000 (radii computed only for the points the stored k-th distances let a
    # query reach); the learned budget's levels are 5 / 10 proxies from a beam of
    # 100 (this size needs more proxies than the 1M mixture).
    "large-10M-d96-K200": dict(n=10_000_000, d=96, C=1024, sigma=1.0, seed=4, dirichlet=False, nq=100_000,
                               qseed=1004, M=16, efc=200, K=200, iters=10, S=50, k=10, Kp=200, ef=200,
                               m_sweep=[1, 2, 3, 4, 5, 6, 8, 10, 15, 20, 50], gt_subset=5000, val_n=4000,
                               budget_levels=(5, 10, 100)),
    # Learned search budget: 1M x 256, 512 equal Gaussians (sigma 1.5, seed 3),
    # K_knng=500; the MLP trained on 200,000 seeded queries (draw seed 1003) labelled
    # by the method itself, evaluated on 20,000 held-out queries (draw seed 2003);
    # the caller's m is 50 and the budget falls back to it below confidence 0.9.
    "learned-1M-d256-K500": dict(n=1_000_000, d=256, C=512, sigma=1.5, seed=3, dirichlet=False, nq=20_000,
                                 qseed=2003, tseed=1003, M=16, efc=400, K=500, iters=10, S=50, k=10, Kp=500,
                                 ef=200, m_sweep=[50], fixed_m=50, fixed_conf=0.9, budget_levels=(3, 10, 0)),
    # Batched uneven queries + dynamic inserts: the 1M mixture split 0.5 by the
    # reference's permutation (std::shuffle, mt19937(42)); build on 500k, insert
    # 500k in 10 batches of 50k (insertPointDynamic with m_update proxies), flat
    # reverse CSR, then 10,000 queries per step with m ~ U{1..50}, ef_search ~
    # U[50, 400] (parameter seed 7), K'=500, k=10, replayed from a captured plan.
    "dynamic-1M-d128-K500": dict(n=1_000_000, d=128, C=256, sigma=1.0, seed=2, dirichlet=True, nq=10_000,
                                 qseed=1002, M=16, efc=400, K=500, iters=10, S=50, k=10, Kp=500, ef=200,
                                 m_sweep=[5], split=0.5, batches=10, m_update=10, bidirectional=False,
                                 m_range=(1, 50), ef_range=(50, 400), pseed=7),
    # The same protocol at the reference's CPU-runnable size (100k x 128, K_knng=100):
    # the reference's own dynamic inserts run beside the GPU's on it.
    "dynamic-100k-d128-K100": dict(n=100_000, d=128, C=64, sigma=1.0, seed=0, dirichlet=False, nq=1_000, qseed=1,
                                   M=16, efc=400, K=100, iters=10, S=50, k=10, Kp=100, ef=200, m_sweep=[5],
                                   split=0.5, batches=10, m_update=10, bidirectional=False,
                                   m_range=(1, 50), ef_range=(50, 400), pseed=7),
    # The reference's CPU-runnable case: 100k x 128, 64 equal Gaussians (seed 0), K_knng=100.
    "plain-100k-d128-K100": dict(n=100_000, d=128, C=64, sigma=1.0, seed=0, dirichlet=False, nq=1_000, qseed=1,
                                 M=16, efc=400, K=100, iters=10, S=50, k=10, Kp=100, ef=200,
                                 m_sweep=[1, 2, 3, 4, 5, 6, 8, 10, 20, 50]),
}
TARGET_RECALL = 0.95


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), float(j["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def start(self):
        def run():
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                         timeout=5).stdout.strip()
                    if out:
                        self.rows.append([x.strip() for x in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)

        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ---------------------------------------------------------------------------
# Seeded synthetic inputs: Gaussian mixtures with the benchmark shapes (centres ~
# N(0, 4 I) from default_rng(centre_seed), equal or Dirichlet(1) weights, points
# = centre + N(0, sigma^2 I), float32).  The RkNN ground truth comes from
# hrnn_b200.groundtruth (float64 decisions on the GPU).
# ---------------------------------------------------------------------------

def mixture(n: int, d: int, C: int, sigma: float, centre_seed: int, draw_seed: int,
            dirichlet: bool = False) -> np.ndarray:
    rc = np.random.default_rng(centre_seed)
    centres = rc.normal(0.0, 2.0, (C, d))
    w = rc.dirichlet(np.ones(C)) if dirichlet else np.full(C, 1.0 / C)
    r = np.random.default_rng(draw_seed)
    lab = r.choice(C, size=n, p=w)
    return (centres[lab] + r.normal(0.0, sigma, (n, d))).astype(np.float32)


def max_over_ranks(torch, value: float, device, world: int) -> float:
    """Replicas report the slowest rank's time (every rank takes part)."""
    if world <= 1:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_queries(W: dict, rank: int) -> np.ndarray:
    """Each replica answers its own query stream (draw seed offset by the rank)."""
    return mixture(W["nq"], W["d"], W["C"], W["sigma"], W["seed"], W["qseed"] + rank, dirichlet=W["dirichlet"])


VALIDATION_SEED_OFFSET = 5003  # the validation stream: neither timed nor used for training


def validation_queries(W: dict, n: int = 5000) -> np.ndarray:
    """Queries on which the bench makes its parameter choices (the same mixture,
    a draw seed of its own)."""
    return mixture(min(n, W["nq"]), W["d"], W["C"], W["sigma"], W["seed"], W["qseed"] + VALIDATION_SEED_OFFSET,
                   dirichlet=W["dirichlet"])


def kth_radius_fp64(torch, X, k, dev):
    from hrnn_b200 import groundtruth
    return groundtruth.kth_radius_fp64(X, k, dev)


def rknn_gt_fp64(torch, X, Q, kth, dev):
    from hrnn_b200 import groundtruth
    return [np.sort(ids) for ids, _ in groundtruth.rknn_fp64(X, Q, kth, dev)]


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of the search kernels
# per unit of work -- per beam distance for the beam search, per posting for the
# verification -- from an ncu capture of the bench command on the 500k x 128
# profiling case (the 1M index's capture would exceed the few GB a capture may
# hold), keyed by (precision form, phase) and tied to the kernel sources it was
# captured on: the bench line scales it by the units of its own launch, and
# reports none when the sources have changed since (SEARCH_SOURCES hash differs).
NCU_TRAFFIC = {
    "src_hash": "3d3f921bb1720653",
    "command": ("ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum,gpu__time_duration.sum --nvtx "
                "--nvtx-include timed/ -k regex:k_phase_a_fast|k_verify_chunks python bench.py --workload "
                "mixed-500k-d128-K250 --queries 10000 --no-learned --no-cpu-baseline --steps 1 --warmup 3"),
    # bytes per beam distance (phase a) / per posting (phase bc): 842.9 MB over 35.72 M
    # distances (INT8 beam), 1,101.0 MB over 43.83 M postings (streaming verification),
    # 2,854.9 MB over 35.72 M distances (BF16 beam)
    "per_unit": {("int8", "a"): 23.60, ("int8", "bc"): 25.12, ("bf16", "a"): 79.93},
}
SEARCH_SOURCES = ("common.cuh", "beam.cuh", "beam_fast.cuh", "search_plain.cu", "search_bc.cu", "verify_stream.cu",
                  "mixed.cu", "budget.cu")


def search_src_hash() -> str:
    import hashlib
    hsh = hashlib.sha256()
    for f in SEARCH_SOURCES:
        with open(os.path.join(ROOT, "hrnn_b200", "csrc", f), "rb") as fh:
            hsh.update(fh.read())
    return hsh.hexdigest()[:16]


def ncu_traffic(form, phase, st):
    """(DRAM bytes of one launch of that phase's kernel: the capture's bytes per
    unit times this launch's units, source note); (None, why) when not captured on
    the current kernel sources."""
    if not NCU_TRAFFIC:
        return None, "no capture of the current kernels"
    if NCU_TRAFFIC["src_hash"] != search_src_hash():
        return None, f"capture {NCU_TRAFFIC['src_hash']} predates the current kernel sources"
    per_unit = NCU_TRAFFIC["per_unit"].get((form, phase))
    if per_unit is None:
        return None, "form not captured"
    units = st["n_dist"] if phase == "a" else st["n_posting"]
    return int(per_unit * units), (f"ncu dram__bytes_read.sum + dram__bytes_write.sum per "
                                   f"{'beam distance' if phase == 'a' else 'posting'} on {NCU_TRAFFIC['command']} "
                                   f"(kernel sources {NCU_TRAFFIC['src_hash']}), times this launch's units")


def knng_quality(torch, h, X, K, dev, sample=1000, seed=5):
    """Recall of the KNN graph against exact kNN, and the relative error of its
    stored FP32 distances against FP64 ones, on `sample` seeded nodes (FP64 on the
    device; internal ids are data indices, the build inserts in data order)."""
    ids, dists, cnt = h.get_knng()
    n = X.shape[0]
    S = np.sort(np.random.default_rng(seed).choice(n, min(sample, n), replace=False))
    Xd = torch.from_numpy(X).to(dev, torch.float64)
    nx = (Xd * Xd).sum(1)
    rec, errs = [], []
    for c0 in range(0, len(S), 250):
        sl = torch.from_numpy(S[c0:c0 + 250].astype(np.int64)).to(dev)
        xs = Xd[sl]
        D = nx[sl][:, None] - 2.0 * (xs @ Xd.T) + nx[None, :]
        D[torch.arange(len(sl), device=dev), sl] = float("inf")
        exact = torch.topk(D, K, dim=1, largest=False).indices.cpu().numpy()
        for r, u in enumerate(S[c0:c0 + 250]):
            c = int(cnt[u])
            rec.append(len(np.intersect1d(exact[r], ids[u, :c])) / K)
            nb = torch.from_numpy(ids[u, :c].astype(np.int64)).to(dev)
            d64 = ((Xd[nb] - xs[r][None, :]) ** 2).sum(1).cpu().numpy()
            d32 = dists[u, :c].astype(np.float64)
            errs.append(np.abs(d32 - d64) / np.maximum(d64, 1e-300))
        del D
    e = np.concatenate(errs) if errs else np.zeros(1)
    return {"recall_at_K": round(float(np.mean(rec)), 5), "nodes_sampled": int(len(S)),
            "dist_rel_err_max": float(e.max()), "dist_rel_err_mean": float(e.mean())}


def macro_recall(gt, res) -> float:
    s, c = 0.0, 0
    for g, r in zip(gt, res):
        if len(g) == 0:
            continue
        s += len(np.intersect1d(g, np.asarray(r, dtype=np.uint32))) / len(g)
        c += 1
    return s / c if c else 0.0


# ---------------------------------------------------------------------------

class StdoutToStderr:
    """The library prints the reference's progress lines on stdout (hrnn.h:1855);
    the bench keeps stdout for its one JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)

    def __exit__(self, *a):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def build_index(H, W, X, dev_sync, join="exact"):
    with StdoutToStderr():
        return _build_index(H, W, X, dev_sync, join)


def _build_index(H, W, X, dev_sync, join):
    h = H.HRNN(W["d"], W["n"], W["M"], W["efc"], 100, W["K"])
    h.set_join_mode({"exact": H.JOIN_EXACT, "tensor": H.JOIN_TENSOR, "audit": H.JOIN_AUDIT}[join])
    t0 = time.perf_counter()
    h.add_points(X)
    dev_sync()
    t1 = time.perf_counter()
    h.refineKNNG(W["iters"], W["S"])
    dev_sync()
    t2 = time.perf_counter()
    h.buildRKNNG()
    dev_sync()
    t3 = time.perf_counter()
    return h, {"hnsw_insert_s": t1 - t0, "nndescent_s": t2 - t1, "rknng_csr_s": t3 - t2,
               "knng_build_s": t3 - t1}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mixed-1M-d128-K500", choices=list(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=2000, help="queries in the CPU-baseline sample")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-budget form")
    ap.add_argument("--build-only", action="store_true", help="build the index, print its build times, exit")
    ap.add_argument("--budget-train", type=int, default=200_000, help="training queries of the budget MLP")
    ap.add_argument("--budget-levels", default="", help="m0,m1,ef of the learned budget's levels "
                                                         "(ef 0: the caller's beam; default: the workload's)")
    ap.add_argument("--queries", type=int, default=0, help="queries per step (default: the workload's)")
    ap.add_argument("--learned-precision", default="auto", choices=["auto", "bf16", "int8"],
                    help="reduced-precision form the learned budget runs on (auto: the faster one as timed)")
    ap.add_argument("--join", default="exact", choices=["exact", "tensor", "audit"],
                    help="refineKNNG local join: exact FP32 (default), tensor-core screened, or audited screen")
    args = ap.parse_args()
    W = dict(WORKLOADS[args.workload])
    if args.queries > 0:
        W["nq"] = args.queries

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference" and rank != 0:
        return  # the reference arm runs on rank 0 alone

    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    import hrnn_b200 as H
    def dev_sync():
        torch.cuda.synchronize(dev)

    if args.workload.startswith("dynamic-"):
        run_dynamic(args, W, H, torch, dev, dev_sync, rank, world, local)
        if world > 1:
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        return

    t_gen = time.perf_counter()
    X = mixture(W["n"], W["d"], W["C"], W["sigma"], W["seed"], W["seed"], dirichlet=W["dirichlet"])
    Q = replica_queries(W, rank)
    log(f"[bench] data {X.shape} queries {Q.shape} ({time.perf_counter() - t_gen:.1f}s)")

    h, build = build_index(H, W, X, dev_sync, args.join)
    rs = h.last_refine_stats()
    log(f"[bench] build: {json.dumps(build)}")
    build["knng_quality"] = knng_quality(torch, h, X, W["K"], dev)
    log(f"[bench] KNN graph: {json.dumps(build['knng_quality'])}")
    if args.build_only:
        if rank == 0:
            print(json.dumps({"workload": args.workload, "build": build,
                              "refine": {k_: rs[k_] for k_ in ("ms", "sample_ms", "join_ms", "bucket_ms", "merge_ms",
                                                               "proposals", "join_dists", "updates", "screen_survivors",
                                                               "screen_dense_nodes", "join_mode")}}), flush=True)
        return

    # ---- ground truth and the recall sweep (untimed) ----
    # Every parameter choice (the smallest m reaching the recall target per form,
    # the learned budget's confidence and fallback m) is made on a separate
    # validation stream; recall is reported on the timed queries themselves.
    t_gt = time.perf_counter()
    Qv = validation_queries(W, W.get("val_n", 5000))
    if "gt_subset" in W:
        # every point's radius is out of reach at this size: an upper bound of it
        # (the stored k-th distance, widened past FP32 rounding) screens the points
        # some query can reach, and only those get their exact float64 radius
        from hrnn_b200 import groundtruth
        up = h.get_kdist(W["k"]).astype(np.float64) * (1.0 + 1e-4)
        ns = min(W["gt_subset"], len(Q))
        g_, nr = groundtruth.rknn_fp64_bounded(X, np.concatenate([Q[:ns], Qv]), up, W["k"], dev)
        gt, gtv = [np.sort(i) for i, _ in g_[:ns]], [np.sort(i) for i, _ in g_[ns:]]
        build["ground_truth"] = {"queries_with_gt": ns, "validation_queries": len(Qv), "radii_computed": nr}
    else:
        kth = kth_radius_fp64(torch, X, W["k"], dev)
        gt = rknn_gt_fp64(torch, X, Q, kth, dev)
        gtv = rknn_gt_fp64(torch, X, Qv, kth, dev)
    log(f"[bench] fp64 ground truth ({time.perf_counter() - t_gt:.1f}s), mean |RkNN| "
        f"{np.mean([len(g) for g in gt]):.2f}, empty {sum(len(g) == 0 for g in gt)}; validation {len(Qv)} queries")
    # GT ids are data indices; index labels are data indices too.
    nq, d = Q.shape
    forms = {"plain": H.PREC_FP32_EXACT, "mixed": H.PREC_BF16}
    if d % 16 == 0 and d <= 256:
        forms["mixed_int8"] = H.PREC_INT8

    def sweep_form(prec, stop=False):
        """Recall on the validation stream per m; the smallest m reaching the target."""
        h.set_precision(prec)
        sw, mstar = {}, None
        for m in W["m_sweep"]:
            res = h.search_rknn_batch(Qv, m, W["Kp"], W["ef"], threshold=1.0, k=W["k"])
            sw[m] = macro_recall(gtv, res)
            if mstar is None and sw[m] >= TARGET_RECALL:
                mstar = m
                if stop:
                    break
        return sw, (mstar if mstar is not None else W["m_sweep"][-1])

    sweeps, mstars = {}, {}
    for name, prec in forms.items():
        if "fixed_m" in W:  # the workload states the caller's m
            sweeps[name], mstars[name] = {}, W["fixed_m"]
            continue
        sweeps[name], mstars[name] = sweep_form(prec)
        log(f"[bench] {name}: validation recall sweep "
            f"{json.dumps({k_: round(v_, 4) for k_, v_ in sweeps[name].items()})} -> m={mstars[name]}")
    h.set_precision(H.PREC_FP32_EXACT)
    params = {"m": mstars["plain"], "K_prime": W["Kp"], "ef_search": W["ef"], "k": W["k"], "threshold": 1.0}

    if args.impl == "reference":
        run_reference_arm(args, W, h, Q, params, sweeps["plain"], build)
        return

    # ---- timed device steps, per form ----
    # A stream of its own for every timed launch and its events: the library runs
    # a call given the null handle on the index's own (non-blocking) stream, which
    # events on torch's default stream would not order against.
    stream = torch.cuda.Stream(dev)
    hbm, bf16, peak_kind = load_peaks()
    maxM0 = 2 * W["M"]
    qsets = {}
    for qn, (QQ, GG) in {"timed": (Q, gt), "val": (Qv, gtv)}.items():
        nn_ = QQ.shape[0]
        qsets[qn] = {"n": nn_, "gt": GG, "q": torch.from_numpy(QQ).to(dev),
                     "kp": torch.full((nn_,), W["Kp"], dtype=torch.int32, device=dev),
                     "ef": torch.full((nn_,), W["ef"], dtype=torch.int32, device=dev),
                     "off": torch.zeros(nn_ + 1, dtype=torch.int64, device=dev),
                     "lab": torch.zeros(nn_ * 512, dtype=torch.int64, device=dev), "cap": nn_ * 512}

    def timed(prec, m_star, learned=False, steps=None, name=None, qset="timed"):
        """Times `steps` batch calls on the query set (after the warm-up calls);
        the recall reported is that of the timed calls' answers."""
        steps = steps or args.steps
        S = qsets[qset]
        nq_ = S["n"]
        clocks = ClockSampler(local)
        h.set_precision(prec)
        if learned:
            h.set_budget(True, **BUDGET)
        m_dev = torch.full((nq_,), m_star, dtype=torch.int32, device=dev)
        dev_sync()  # made on the default stream, read on `stream`

        # The batch search recorded once as a CUDA graph over the step's buffers
        # (hrnn_search_plan_*, the serving path: no host synchronisation inside a
        # step), replayed once per step.
        plan = h.search_plan(S["q"].data_ptr(), nq_, m_dev.data_ptr(), S["kp"].data_ptr(), S["ef"].data_ptr(),
                             m_star, W["ef"], 1.0, W["k"], S["off"].data_ptr(), S["lab"].data_ptr(), S["cap"],
                             stream.cuda_stream)
        per_run = plan.kernels()

        def step():
            plan.run(stream.cuda_stream)

        for _ in range(args.warmup):
            step()
        if world > 1:
            torch.distributed.barrier()
        dev_sync()
        clocks.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push("timed")  # profilers select the timed steps with this range
        e0.record(stream)
        launches = 0
        for _ in range(steps):
            step()
            launches += per_run
        e1.record(stream)
        dev_sync()
        torch.cuda.nvtx.range_pop()
        ck = clocks.stop()
        ms = max_over_ranks(torch, e0.elapsed_time(e1), dev, world)
        tot, clamped = plan.result(stream.cuda_stream)
        plan.close()
        offs = S["off"].cpu().numpy()
        labs = S["lab"][:tot].cpu().numpy()
        recall = macro_recall(S["gt"], [labs[offs[i]:offs[i + 1]] for i in range(nq_)])
        # counts and per-phase times of the same search: stream-ordered batch calls
        # after the timed steps (the first sizes the batch path's work buffers; the
        # last one's statistics are kept, and its answers must equal the plan's)
        for _ in range(2):
            tot_b = h.search_rknn_batch_device(S["q"].data_ptr(), nq_, m_dev.data_ptr(), S["kp"].data_ptr(),
                                               S["ef"].data_ptr(), 1.0, W["k"], S["off"].data_ptr(),
                                               S["lab"].data_ptr(), S["cap"], stream.cuda_stream)
        st = h.last_search_stats()
        if tot_b != tot or clamped or not np.array_equal(S["off"].cpu().numpy(), offs):
            raise RuntimeError(f"bench: plan and batch call disagree ({tot} vs {tot_b} results, clamped {clamped})")
        # algorithmic bytes of the two phases: rows of 4 bytes/element (FP32), 2 (BF16)
        # or 1 plus 16 bytes of scale / error terms (INT8); the k-distance of each
        # verified id; the FP32 rows of the screens' undecided ids
        rb, rm = {H.PREC_FP32_EXACT: (4, 0), H.PREC_BF16: (2, 4), H.PREC_INT8: (1, 16)}[prec]
        bytes_a = st["n_dist"] * (d * rb + rm) + st["n_expanded"] * (4 + 4 * maxM0)
        bytes_bc = st["n_posting"] * 4 + st["n_verified"] * (d * rb + rm + 4) + \
            st["n_fp32_decided"] * d * 4 + st["n_result"] * 8
        phases = {"phase_a_beam_search": (st["phase_a_ms"], bytes_a),
                  "phase_bc_posting_verify": (st["phase_c_ms"], bytes_bc)}
        dom = max(phases, key=lambda k_: phases[k_][0])
        tms, tb = phases[dom]
        achieved = tb / (tms / 1e3) / 1e9 if tms > 0 else 0.0
        form = {H.PREC_FP32_EXACT: "fp32", H.PREC_BF16: "bf16", H.PREC_INT8: "int8"}[prec]
        traffic, traffic_src = ncu_traffic(form, "a" if dom.startswith("phase_a") else "bc", st)
        roof = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(achieved / hbm, 4), "peak_source": peak_kind, "traffic": traffic,
                "traffic_source": traffic_src,
                "algorithmic_bytes_per_launch": int(tb), "launch_ms": round(tms, 3),
                "per_query": {k_: round(st[k_] / nq_, 3) for k_ in
                              ("n_dist", "n_expanded", "n_posting", "n_verified", "n_result", "n_lowp_decided",
                               "n_fp32_decided", "n_fp64_decided", "n_fp64_flipped")},
                "phase_ms": {"a": round(st["phase_a_ms"], 3), "b": round(st["phase_b_ms"], 3),
                             "c": round(st["phase_c_ms"], 3)}}
        if learned:
            roof["budget_levels"] = st["n_budget"]
            h.set_budget(False, **BUDGET)
        return {"qps": world * nq_ * steps / (ms / 1e3), "ms_per_step": ms / steps, "launches": launches,
                "roofline": roof, "clocks": ck, "m": m_star, "prec": prec, "recall_sweep": sweeps[name],
                "recall": recall}

    results = {}
    for name, prec in forms.items():
        results[name] = timed(prec, mstars[name], name=name)

    # ---- learned search budget on the faster reduced-precision form: trained on
    # separate seeded queries (untimed), then the fastest (confidence, fallback m)
    # pair reaching the recall target ----
    budget_info = None
    if not args.no_learned:
        if args.learned_precision == "auto":
            lp = max((f for f in forms if f != "plain"), key=lambda f: results[f]["qps"])
        else:
            lp = {"bf16": "mixed", "int8": "mixed_int8"}[args.learned_precision]
            if lp not in forms:
                lp = "mixed"
        lprec = forms[lp]
        if args.budget_levels:
            m0_, m1_, ef_ = (int(x) for x in args.budget_levels.split(","))
            BUDGET.update(m0=m0_, m1=m1_, ef=ef_)
        elif "budget_levels" in W:
            BUDGET.update(dict(zip(("m0", "m1", "ef"), W["budget_levels"])))
        budget_info = train_budget(H, h, W, args, dev_sync, lprec, mstars["plain"])
        budget_info["precision_form"] = lp
        cands = []
        for c in ([W["fixed_conf"]] if "fixed_conf" in W else CONFIDENCES):
            if "fixed_m" in W:  # the workload states the fallback m and the cutoff
                cands.append((c, W["fixed_m"], {}))
                continue
            BUDGET["confidence"] = c
            h.set_budget(True, **BUDGET)
            sw, mstar = sweep_form(lprec, stop=True)
            log(f"[bench] learned (confidence {c}): recall sweep (fallback m) "
                f"{json.dumps({k_: round(v_, 4) for k_, v_ in sw.items()})} -> m={mstar}")
            if sw[mstar] >= TARGET_RECALL:
                cands.append((c, mstar, sw))
        h.set_budget(False, **BUDGET)
        h.set_precision(H.PREC_FP32_EXACT)
        trial = []
        for c, mstar, sw in cands:  # timed on the validation stream
            BUDGET["confidence"] = c
            sweeps["learned"] = sw
            r = timed(lprec, mstar, learned=True, steps=3, name="learned", qset="val")
            trial.append({"confidence": c, "m": mstar, "recall_val": round(r["recall"], 4),
                          "value_val": round(r["qps"], 1)})
        budget_info["candidates"] = trial
        if "fixed_conf" not in W:
            trial = [t_ for t_ in trial if t_["recall_val"] >= TARGET_RECALL]
        if trial:
            best = max(trial, key=lambda t_: t_["value_val"])
            BUDGET["confidence"] = best["confidence"]
            sweeps["learned"] = next(sw for c, _, sw in cands if c == best["confidence"])
            mstars["learned"] = best["m"]
            budget_info["confidence"] = best["confidence"]
            results["learned"] = timed(lprec, mstars["learned"], learned=True, name="learned")
    head = max(results, key=lambda k_: results[k_]["qps"])
    R = results[head]
    qps, ms_per_step, launches, roofline, ck = R["qps"], R["ms_per_step"], R["launches"], R["roofline"], R["clocks"]
    m_star = R["m"]
    log("[bench] " + ", ".join(f"{k_} {r_['qps']:.0f} q/s (m={r_['m']})" for k_, r_ in results.items()))

    # ---- end to end through the host-buffer entry point (headline form) ----
    h.set_precision(R["prec"])
    if head == "learned":
        h.set_budget(True, **BUDGET)
    # Pinned host buffers; every step copies the queries and their (m, K', ef) in,
    # searches, copies the offsets and the labels out and waits: one call of the
    # C ABI's hrnn_search_plan_run_host on a plan made for the batch shape (the
    # serving path; plan creation is setup, outside the timed region).  The
    # one-call batch entry point hrnn_search_rknn_batch on the same host buffers
    # is timed beside it.
    e2e_steps = max(1, args.steps)
    q_pin = torch.from_numpy(np.ascontiguousarray(Q)).pin_memory()
    p_m = torch.full((nq,), m_star, dtype=torch.int32).pin_memory()
    p_kp = torch.full((nq,), W["Kp"], dtype=torch.int32).pin_memory()
    p_ef = torch.full((nq,), W["ef"], dtype=torch.int32).pin_memory()
    p_off = torch.zeros(nq + 1, dtype=torch.int64).pin_memory()
    e2e_cap = nq * 512
    p_lab = torch.zeros(e2e_cap, dtype=torch.int64).pin_memory()
    d_in = {"q": torch.zeros((nq, d), dtype=torch.float32, device=dev),
            **{k_: torch.zeros(nq, dtype=torch.int32, device=dev) for k_ in ("m", "kp", "ef")},
            "off": torch.zeros(nq + 1, dtype=torch.int64, device=dev),
            "lab": torch.zeros(e2e_cap, dtype=torch.int64, device=dev)}
    dev_sync()  # made on the default stream, written on `stream`
    e2e_plan = h.search_plan(d_in["q"].data_ptr(), nq, d_in["m"].data_ptr(), d_in["kp"].data_ptr(),
                             d_in["ef"].data_ptr(), m_star, W["ef"], 1.0, W["k"], d_in["off"].data_ptr(),
                             d_in["lab"].data_ptr(), e2e_cap, stream.cuda_stream)

    def e2e_step():
        return e2e_plan.run_host(q_pin.data_ptr(), p_m.data_ptr(), p_kp.data_ptr(), p_ef.data_ptr(),
                                 p_off.data_ptr(), p_lab.data_ptr(), e2e_cap, stream.cuda_stream)[0]

    def e2e_batch_step():
        return h.search_rknn_batch_host(q_pin.data_ptr(), nq, p_m.data_ptr(), p_kp.data_ptr(), p_ef.data_ptr(), 1.0,
                                        W["k"], p_off.data_ptr(), p_lab.data_ptr(), e2e_cap)

    e2e_batch = None
    for fn in (e2e_batch_step, e2e_step):  # the plan's run last: its answers are read below
        for _ in range(max(1, args.warmup)):
            fn()
        dev_sync()
        t0 = time.perf_counter()
        total_res = 0
        for _ in range(e2e_steps):
            total_res = fn()
        e2e_s = max_over_ranks(torch, time.perf_counter() - t0, dev, world)
        if fn is e2e_batch_step:
            e2e_batch = round(world * nq * e2e_steps / e2e_s, 1)
    e2e_plan.close()
    e2e = {"value": world * nq * e2e_steps / e2e_s, "unit": "queries/s",
           "h2d_bytes_per_step": int(nq * d * 4 + 3 * nq * 4), "d2h_bytes_per_step": int((nq + 1) * 8 + total_res * 8),
           "host_buffers": "pinned", "call": "hrnn_search_plan_run_host",
           "batch_call_value": e2e_batch, "batch_call": "hrnn_search_rknn_batch"}
    offs = p_off.numpy().astype(np.int64)
    labs = p_lab.numpy()[:total_res]
    out = [labs[offs[i]:offs[i + 1]] for i in range(nq)]
    recall_timed = macro_recall(gt, out)
    h.set_precision(H.PREC_FP32_EXACT)
    if head == "learned":
        h.set_budget(False, **BUDGET)
    params = {"m": m_star, "K_prime": W["Kp"], "ef_search": W["ef"], "k": W["k"], "threshold": 1.0}
    sweep = sweeps[head]

    # ---- NNDescent roofline, per iteration: the lists read and written once
    # (2 N K 8), every node's sample rows gathered once in FP32, every proposal
    # (target, source, d) written once and read once (24 bytes).  The exact re-rank
    # of the screened pairs reads the rows already staged on chip, so it moves no
    # HBM bytes.  (Charging each proposal two FP32 rows from HBM instead,
    # proposals * (8 + 2 d 4), gives the "per_proposal_rows" figure.) ----
    it_bytes, it_bytes_rows = [], []
    for i in range(rs["iters"]):
        base = 2 * W["n"] * W["K"] * 8 + rs["sample_entries"][i] * d * 4
        it_bytes.append(base + rs["proposals"][i] * 24)
        it_bytes_rows.append(base + rs["proposals"][i] * (8 + 2 * d * 4))
    nnd_ms = sum(rs["ms"])
    build["nndescent_iter_ms"] = [round(x, 2) for x in rs["ms"]]
    build["nndescent_phase_ms"] = {k_: [round(x, 2) for x in rs[k_ + "_ms"]] for k_ in ("sample", "join", "bucket", "merge")}
    build["nndescent_roofline"] = {"bound": "hbm", "achieved": round(sum(it_bytes) / (nnd_ms / 1e3) / 1e9, 1)
                                   if nnd_ms > 0 else None, "peak": hbm, "unit": "GB/s",
                                   "frac": round(sum(it_bytes) / (nnd_ms / 1e3) / 1e9 / hbm, 4) if nnd_ms else None,
                                   "bytes_per_iter": it_bytes,
                                   "per_proposal_rows_frac": round(sum(it_bytes_rows) / (nnd_ms / 1e3) / 1e9 / hbm, 4)
                                   if nnd_ms else None,
                                   "join_dists": rs["join_dists"], "proposals": rs["proposals"],
                                   "join_mode": rs["join_mode"], "screen_survivors": rs["screen_survivors"],
                                   "screen_dense_nodes": rs["screen_dense_nodes"]}

    cpu, parity = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # Parity on this index: the plain form's answers for the CPU sample at the
        # plain form's parameters, and the headline form's answers (from the e2e
        # leg) whose every point the reference's own FP32 test must accept.
        ns = min(args.cpu_sample, nq)
        pparams = dict(params, m=mstars["plain"])
        h.set_precision(H.PREC_FP32_EXACT)
        plain_ans = h.search_rknn_batch(Q[:ns], pparams["m"], W["Kp"], W["ef"], threshold=1.0, k=W["k"])
        kd_all = h.get_kdist(W["k"])  # kdist(p, k-1), FLT_MAX where the list is shorter (hrnn.h:286-293)
        cpu, parity = cpu_baseline(h, W, Q, pparams, ns, gt=gt[:ns], plain_ans=plain_ans, head_ans=out[:ns],
                                   head=head, X=X, kcol=kd_all)
        del h
        cpu["build"] = cpu_build_baseline(H, torch, dev, dev_sync)
        log(f"[bench] build baseline: {json.dumps(cpu['build'])}")

    line = {
        "metric": "RkNN queries/s at recall>=0.95 (k=10)", "value": round(qps, 1), "unit": "queries/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {H.PREC_FP32_EXACT: "f32", H.PREC_BF16: "bf16 screen + f32/f64 decisions",
                  H.PREC_INT8: "int8 beam; int8/bf16 screens + f32/f64 decisions"}[R["prec"]] +
                 ("; bf16 budget MLP" if head == "learned" else ""),
        "data": "synthetic (seeded Gaussian mixture)",
        "config": {"workload": args.workload, "n": W["n"], "dim": d, "K_knng": W["K"], "M": W["M"],
                   "ef_construction": W["efc"], "queries_per_step": nq, "form": head,
                   **params, "recall_macro": round(recall_timed, 4),
                   "recall_sweep_validation": {str(k_): round(v, 4) for k_, v in sweep.items()},
                   "selection": "m (and the learned budget's confidence) chosen on a separate validation stream "
                                "of seeded queries; recall_macro is that of the timed queries' answers",
                   "parallelism": f"replicas{world}", "l2_flush": "inputs larger than L2 (index 7 GB)"},
        "forms": {k_: {"value": round(r_["qps"], 1), "ms_per_step": round(r_["ms_per_step"], 3), "m": r_["m"],
                       "recall_macro": round(r_["recall"], 4), "clocks": r_["clocks"],
                       "recall_sweep_validation": {str(a_): round(b_, 4) for a_, b_ in r_["recall_sweep"].items()},
                       "roofline": r_["roofline"]} for k_, r_ in results.items()},
        "speedup_vs_plain": round(qps / results["plain"]["qps"], 3),
        "learned_budget": budget_info,
        "e2e": {k_: (round(v, 1) if isinstance(v, float) else v) for k_, v in e2e.items()},
        "gpu_launches": int(launches), "roofline": roofline, "cpu_baseline": cpu, "parity": parity, "clocks": ck,
        "knng_build": {k_: (round(v, 3) if isinstance(v, float) else v) for k_, v in build.items()},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


# ---------------------------------------------------------------------------
# Batched uneven queries after dynamic inserts (the dynamic-* workloads)
# ---------------------------------------------------------------------------

def uneven_params(W: dict, nq: int):
    """Per-query m ~ U{m_range}, ef_search ~ U[ef_range] (seeded), K' and k fixed."""
    r = np.random.default_rng(W["pseed"])
    m = r.integers(W["m_range"][0], W["m_range"][1] + 1, nq).astype(np.uint32)
    ef = r.integers(W["ef_range"][0], W["ef_range"][1] + 1, nq).astype(np.uint32)
    return m, np.full(nq, W["Kp"], np.uint32), ef


def dynamic_build(H, W, X, dev_sync, perm, ref=False, threads=1):
    """The reference's dynamic protocol (src/hrnn_dynamic_test.cpp:200-203, 240-262,
    268-288, 305-331, 368): build on the first split of the permutation (labels =
    data indices), refineKNNG, buildRKNNG_mutable, insertPointDynamic for the rest
    in batches, then the flat reverse CSR the search reads.  ref=True runs the
    reference's own code (oracle/_ref) with `threads` host threads instead."""
    n = W["n"]
    split = int(n * W["split"])
    base, ins = perm[:split].astype(np.uint64), perm[split:].astype(np.uint64)
    t = {}
    with StdoutToStderr():
        if ref:
            from oracle import ref as R
            h = R.RefIndex.create(W["d"], n, W["M"], W["efc"], 100, W["K"])
        else:
            h = H.HRNN(W["d"], n, W["M"], W["efc"], 100, W["K"])
        t0 = time.perf_counter()
        if ref:
            h.add_points(X[base.astype(np.int64)], labels=base, threads=threads)
        else:
            h.add_points(X[base.astype(np.int64)], labels=base)
        dev_sync()
        t1 = time.perf_counter()
        if ref:
            h.refine(W["iters"], W["S"], threads=threads)
            h.build_mutable()
        else:
            h.refineKNNG(W["iters"], W["S"])
            h.buildRKNNG_mutable()
        dev_sync()
        t2 = time.perf_counter()
        nb = W["batches"]
        per = (len(ins) + nb - 1) // nb
        batch_ms, dyn = [], []
        for b in range(nb):
            sl = ins[b * per:(b + 1) * per]
            if len(sl) == 0:
                continue
            tb = time.perf_counter()
            if ref:
                h.insert_dynamic(X[sl.astype(np.int64)], sl, m_update=W["m_update"],
                                 bidirectional=W["bidirectional"], threads=threads)
            else:
                h.insertPointDynamic(X[sl.astype(np.int64)], sl, W["m_update"], W["bidirectional"])
            dev_sync()
            batch_ms.append(round((time.perf_counter() - tb) * 1e3, 2))
            if not ref:
                dyn.append({k_: (round(v_, 2) if isinstance(v_, float) else v_)
                            for k_, v_ in h.last_dynamic_stats().items()})
        t3 = time.perf_counter()
        if ref:
            h.build_rknng()
        else:
            h.buildRKNNG()
        dev_sync()
        t4 = time.perf_counter()
    t = {"initial_points": int(split), "inserted_points": int(len(ins)), "batches": len(batch_ms),
         "hnsw_insert_s": round(t1 - t0, 3), "refine_and_mutable_s": round(t2 - t1, 3),
         "insert_total_s": round(t3 - t2, 3), "insert_batch_ms": batch_ms,
         "insert_points_per_s": round(len(ins) / max(t3 - t2, 1e-9), 1), "flat_rknng_s": round(t4 - t3, 3),
         "m_update": W["m_update"], "bidirectional": bool(W["bidirectional"])}
    if dyn:
        t["per_batch"] = dyn
    return h, t


def run_dynamic(args, W, H, torch, dev, dev_sync, rank, world, local):
    X = mixture(W["n"], W["d"], W["C"], W["sigma"], W["seed"], W["seed"], dirichlet=W["dirichlet"])
    Q = replica_queries(W, rank)
    nq, d = Q.shape
    perm = H.dynamic_split(W["n"], 42)
    m_h, kp_h, ef_h = uneven_params(W, nq)
    h, dyn = dynamic_build(H, W, X, dev_sync, perm)
    log(f"[bench] dynamic build: {json.dumps({k_: v_ for k_, v_ in dyn.items() if k_ != 'per_batch'})}")
    kth = kth_radius_fp64(torch, X, W["k"], dev)
    gt = rknn_gt_fp64(torch, X, Q, kth, dev)
    if args.impl == "reference":
        run_reference_arm(args, W, h, Q, {"m": m_h, "K_prime": kp_h, "ef_search": ef_h, "k": W["k"],
                                          "threshold": 1.0}, None, dyn)
        return
    # A stream of its own: the captured plan is an asynchronous graph launch, so
    # the timing events must sit on the stream it runs on (a null handle would
    # send the library's calls to the index's own stream).
    stream = torch.cuda.Stream(dev)
    q_d = torch.from_numpy(Q).to(dev)
    m_d = torch.from_numpy(m_h.view(np.int32)).to(dev)
    kp_d = torch.from_numpy(kp_h.view(np.int32)).to(dev)
    ef_d = torch.from_numpy(ef_h.view(np.int32)).to(dev)
    cap = nq * 2048
    off_d = torch.zeros(nq + 1, dtype=torch.int64, device=dev)
    lab_d = torch.zeros(cap, dtype=torch.int64, device=dev)
    dev_sync()  # made on the default stream, read on `stream`
    hbm, _, peak_kind = load_peaks()
    forms = {"plain": H.PREC_FP32_EXACT, "mixed_int8": H.PREC_INT8}
    out = {}
    answers = {}
    for name, prec in forms.items():
        h.set_precision(prec)
        # stream-ordered batch calls
        def step():
            return h.search_rknn_batch_device(q_d.data_ptr(), nq, m_d.data_ptr(), kp_d.data_ptr(), ef_d.data_ptr(),
                                              1.0, W["k"], off_d.data_ptr(), lab_d.data_ptr(), cap,
                                              stream.cuda_stream)
        for _ in range(args.warmup):
            step()
        dev_sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            tot = step()
        e1.record(stream)
        dev_sync()
        ms_b = max_over_ranks(torch, e0.elapsed_time(e1), dev, world)
        st = h.last_search_stats()
        offs, labs = off_d.cpu().numpy(), lab_d[:tot].cpu().numpy()
        ans_b = [labs[offs[i]:offs[i + 1]].copy() for i in range(nq)]
        off_d.zero_()  # the plan's replays must write the answers themselves
        lab_d.zero_()
        dev_sync()
        # the same batch replayed from a captured plan (one graph launch per batch)
        plan = h.search_plan(q_d.data_ptr(), nq, m_d.data_ptr(), kp_d.data_ptr(), ef_d.data_ptr(),
                             W["m_range"][1], W["ef_range"][1], 1.0, W["k"], off_d.data_ptr(), lab_d.data_ptr(), cap,
                             stream.cuda_stream)
        clocks = ClockSampler(local)
        for _ in range(args.warmup):
            plan.run(stream.cuda_stream)
        dev_sync()
        clocks.start()
        e0.record(stream)
        for _ in range(args.steps):
            plan.run(stream.cuda_stream)
        e1.record(stream)
        dev_sync()
        ck = clocks.stop()
        ms_p = max_over_ranks(torch, e0.elapsed_time(e1), dev, world)
        tot_p, clamped = plan.result(stream.cuda_stream)
        plan.close()
        offs, labs = off_d.cpu().numpy(), lab_d[:tot_p].cpu().numpy()
        ans_p = [labs[offs[i]:offs[i + 1]].copy() for i in range(nq)]
        same = sum(np.array_equal(a, b) for a, b in zip(ans_b, ans_p))
        answers[name] = ans_p
        rb, rm = {H.PREC_FP32_EXACT: (4, 0), H.PREC_INT8: (1, 16)}[prec]
        bytes_bc = st["n_posting"] * 4 + st["n_verified"] * (d * rb + rm + 4) + st["n_fp32_decided"] * d * 4 + \
            st["n_result"] * 8
        bytes_a = st["n_dist"] * (d * rb + rm) + st["n_expanded"] * (4 + 4 * 2 * W["M"])
        phases = {"phase_a_beam_search": (st["phase_a_ms"], bytes_a),
                  "phase_bc_posting_verify": (st["phase_c_ms"], bytes_bc)}
        dom = max(phases, key=lambda k_: phases[k_][0])
        tms, tb = phases[dom]
        achieved = tb / (tms / 1e3) / 1e9 if tms > 0 else 0.0
        out[name] = {"value_plan": round(world * nq * args.steps / (ms_p / 1e3), 1),
                     "value_batch_calls": round(world * nq * args.steps / (ms_b / 1e3), 1),
                     "ms_per_step_plan": round(ms_p / args.steps, 3), "ms_per_step_batch": round(ms_b / args.steps, 3),
                     "recall_macro": round(macro_recall(gt, ans_p), 4), "plan_equals_batch_calls": int(same),
                     "clamped": bool(clamped), "clocks": ck,
                     "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": hbm,
                                  "unit": "GB/s", "frac": round(achieved / hbm, 4), "peak_source": peak_kind,
                                  "traffic": None, "algorithmic_bytes_per_launch": int(tb),
                                  "launch_ms": round(tms, 3),
                                  "phase_ms": {"a": round(st["phase_a_ms"], 3), "b": round(st["phase_b_ms"], 3),
                                               "c": round(st["phase_c_ms"], 3)},
                                  "per_query": {k_: round(st[k_] / nq, 2) for k_ in
                                                ("n_dist", "n_expanded", "n_posting", "n_verified", "n_result")}},
                     "a_launch_shape": {"warps_per_block": st["a_warps_per_block"],
                                        "visit_slots": st["a_visit_slots"]}}
        log(f"[bench] {name}: {json.dumps({k_: v_ for k_, v_ in out[name].items() if k_ != 'roofline'})}")
    h.set_precision(H.PREC_FP32_EXACT)
    # end to end: the host-buffer entry point with the per-query arrays
    q_pin = torch.from_numpy(np.ascontiguousarray(Q)).pin_memory()
    pm, pk, pe = (torch.from_numpy(a.view(np.int32)).pin_memory() for a in (m_h, kp_h, ef_h))
    p_off = torch.zeros(nq + 1, dtype=torch.int64).pin_memory()
    p_lab = torch.zeros(cap, dtype=torch.int64).pin_memory()
    for _ in range(max(1, args.warmup)):
        h.search_rknn_batch_host(q_pin.data_ptr(), nq, pm.data_ptr(), pk.data_ptr(), pe.data_ptr(), 1.0, W["k"],
                                 p_off.data_ptr(), p_lab.data_ptr(), cap)
    dev_sync()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        tot = h.search_rknn_batch_host(q_pin.data_ptr(), nq, pm.data_ptr(), pk.data_ptr(), pe.data_ptr(), 1.0,
                                       W["k"], p_off.data_ptr(), p_lab.data_ptr(), cap)
    e2e_s = max_over_ranks(torch, time.perf_counter() - t0, dev, world)
    e2e = {"value": round(world * nq * args.steps / e2e_s, 1), "unit": "queries/s",
           "h2d_bytes_per_step": int(nq * d * 4 + 3 * nq * 4), "d2h_bytes_per_step": int((nq + 1) * 8 + tot * 8),
           "host_buffers": "pinned", "form": "plain"}
    # parity of the plain form's answers with the reference's searchRknn on this index
    parity, cpu = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import ref
        if ref.available():
            import shutil
            td, pth = _save_for_reference(h)
            try:
                r = ref.RefIndex.load(pth, W["d"])
                ns = min(args.cpu_sample, nq)
                cores = os.cpu_count() or 1
                res, secs = r.search_batch(Q[:ns], m_h[:ns], kp_h[:ns], ef_h[:ns], k=W["k"], threads=cores,
                                           return_seconds=True)
                mism = [i for i in range(ns) if not np.array_equal(np.asarray(res[i], np.uint64),
                                                                     np.asarray(answers["plain"][i], np.uint64))]
                parity = {"queries": ns, "mismatches": len(mism), "first_mismatches": mism[:8],
                          "params": "per-query m, ef_search as timed"}
                cpu = {"value": round(ns / secs, 1), "unit": "queries/s", "cores": cores, "kind": "reference",
                       "sample": f"{ns} of the step's queries, {cores} threads"}
                del r
            finally:
                shutil.rmtree(td, ignore_errors=True)
    head = max(out, key=lambda k_: out[k_]["value_plan"])
    line = {
        "metric": "RkNN queries/s (k=10), uneven per-query m and ef_search after dynamic inserts",
        "value": out[head]["value_plan"], "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": out[head]["ms_per_step_plan"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if head == "plain" else "int8 beam/screen + f32/f64",
        "data": "synthetic (seeded Gaussian mixture)",
        "config": {"workload": args.workload, "n": W["n"], "dim": d, "K_knng": W["K"], "M": W["M"],
                   "ef_construction": W["efc"], "queries_per_step": nq, "form": head, "K_prime": W["Kp"],
                   "m": f"U{{{W['m_range'][0]}..{W['m_range'][1]}}}", "ef_search": f"U[{W['ef_range'][0]}, "
                   f"{W['ef_range'][1]}]", "k": W["k"], "recall_macro": out[head]["recall_macro"],
                   "l2_flush": "inputs larger than L2 (index > 3 GB)", "parallelism": f"replicas{world}"},
        "forms": out, "dynamic": dyn, "e2e": e2e, "parity": parity, "cpu_baseline": cpu,
        "roofline": out[head]["roofline"], "clocks": out[head]["clocks"],
    }
    if W["n"] <= 200_000 and rank == 0 and not args.no_cpu_baseline:
        line["reference_dynamic"] = reference_dynamic(H, W, X, Q, gt, m_h, kp_h, ef_h)
    if rank == 0:
        print(json.dumps(line), flush=True)


def reference_dynamic(H, W, X, Q, gt, m_h, kp_h, ef_h):
    """The reference's own dynamic protocol on the same points, permutation and
    queries with all host threads: build, insert and recall beside the GPU's."""
    from oracle import ref
    if not ref.available():
        return {"kind": "reference", "sample": "oracle/_ref not built"}
    cores = os.cpu_count() or 1
    perm = H.dynamic_split(W["n"], 42)
    r, t = dynamic_build(H, W, X, lambda: None, perm, ref=True, threads=cores)
    res, secs = r.search_batch(Q, m_h, kp_h, ef_h, k=W["k"], threads=cores, return_seconds=True)
    t.update({"kind": "reference", "cores": cores, "recall_macro": round(macro_recall(gt, res), 4),
              "search_queries_per_s": round(len(Q) / secs, 1)})
    return t


# Learned budget: level 0 = 3 proxies, level 1 = 5 proxies, both from a beam of 64
# (two-pass mode); a query takes a level when the MLP gives that level's answer
# being complete a probability >= the cutoff, else it continues the search with
# the caller's (m, ef_search).
BUDGET = dict(m0=3, m1=5, ef=64, confidence=0.9)
CONFIDENCES = (0.95, 0.98, 0.99, 0.995, 0.998)
# The labels compare a level's answer with the caller's own answer (m, ef_search):
# a level is "complete" for a query when it returns every point the caller's
# search returns, so taking it changes the work and not the answer.


def _search_sets(h, Q, m, kp, ef, k, chunk=10_000):
    out = []
    for s in range(0, Q.shape[0], chunk):
        out.extend(h.search_rknn_batch(Q[s:s + chunk], m, kp, ef, threshold=1.0, k=k))
    return out


def train_budget(H, h, W, args, dev_sync, prec, label_m):
    """Features and labels of `args.budget_train` seeded queries (a stream separate
    from the timed ones) in the serving precision `prec`, then MLP training on the
    GPU.  A label says whether a level's answer contains the answer of the caller's
    search (label_m proxies, the workload's ef_search)."""
    t0 = time.perf_counter()
    n = args.budget_train
    Qtr = mixture(n, W["d"], W["C"], W["sigma"], W["seed"], W.get("tseed", W["qseed"] + 7919),
                  dirichlet=W["dirichlet"])
    h.set_precision(prec)
    full = _search_sets(h, Qtr, label_m, W["Kp"], W["ef"], W["k"])
    Y = np.zeros((n, 2), np.uint8)
    for j, ml in enumerate((BUDGET["m0"], BUDGET["m1"])):
        got = _search_sets(h, Qtr, ml, W["Kp"], BUDGET["ef"] or W["ef"], W["k"])
        Y[:, j] = [np.isin(f, g, assume_unique=True).all() for f, g in zip(full, got)]
    t1 = time.perf_counter()
    h.set_budget(False, **BUDGET)
    feat = np.concatenate([h.budget_features(Qtr[s:s + 50_000], W["k"], label_m, W["ef"])
                           for s in range(0, n, 50_000)])
    dev_sync()
    t2 = time.perf_counter()
    ho = n // 10  # the last tenth is held out
    loss = h.budget_train(feat[:-ho], Y[:-ho], epochs=30, batch=1024, lr=2e-3, seed=11)
    dev_sync()
    t3 = time.perf_counter()
    z = h.budget_predict(feat[-ho:])
    p = 1.0 / (1.0 + np.exp(-z.astype(np.float64)))
    heldout = []
    for conf in CONFIDENCES:
        take0 = p[:, 0] >= conf
        take1 = ~take0 & (p[:, 1] >= conf)
        wrong = (take0 & (Y[-ho:, 0] == 0)) | (take1 & (Y[-ho:, 1] == 0))
        heldout.append({"confidence": conf, "level_share": [round(float(take0.mean()), 4),
                                                            round(float(take1.mean()), 4)],
                        "wrong_level_rate": round(float(wrong.mean()), 5)})
    h.set_precision(H.PREC_FP32_EXACT)
    info = {"train_queries": n, "levels": {"m0": BUDGET["m0"], "m1": BUDGET["m1"], "ef": BUDGET["ef"] or W["ef"]},
            "label_ref": {"m": label_m, "ef": W["ef"]},
            "label_rate": [round(float(Y[:, 0].mean()), 4), round(float(Y[:, 1].mean()), 4)],
            "final_loss": round(loss, 4), "heldout_queries": ho, "heldout": heldout,
            "labels_s": round(t1 - t0, 1), "features_s": round(t2 - t1, 1), "train_s": round(t3 - t2, 1)}
    log(f"[bench] learned budget: {json.dumps(info)}")
    return info


def _save_for_reference(h):
    td = tempfile.mkdtemp(prefix="hrnn_bench_")
    p = os.path.join(td, "index.idx")
    t0 = time.perf_counter()
    h.saveIndex(p)
    log(f"[bench] saved index for the reference ({os.path.getsize(p) / 1e9:.2f} GB, "
        f"{time.perf_counter() - t0:.1f}s)")
    return td, p


def cpu_baseline(h, W, Q, params, sample, gt=None, plain_ans=None, head_ans=None, head=None, X=None, kcol=None):
    """The reference's searchRknn (oracle/_ref) on the same index on this host's
    cores: all threads on `sample` queries, and one thread (the reference
    protocol, src/hrnn_search.cpp:168-180) on a tenth of them.  Returns
    (baseline, parity): the reference's answers for the sample are compared query
    by query with the GPU plain form's (`plain_ans`, same m, K', ef, k,
    threshold), and every point the headline form returned (`head_ans`) is put
    to the reference's own FP32 test d(q, p) <= kdist(p, k-1) (hrnn.h:2058-2069,
    286-293) with the reference's L2 (space_l2.h)."""
    from oracle import ref
    if not ref.available():
        return ({"value": None, "unit": "queries/s", "cores": 0, "kind": "reference",
                 "sample": "oracle/_ref not built"}, None)
    import shutil
    td, p = _save_for_reference(h)
    try:
        t0 = time.perf_counter()
        r = ref.RefIndex.load(p, W["d"])
        log(f"[bench] reference loaded the index ({time.perf_counter() - t0:.1f}s)")
        cores = os.cpu_count() or 1
        Qs = Q[:sample]
        res, secs = r.search_batch(Qs, params["m"], params["K_prime"], params["ef_search"], k=params["k"],
                                   threads=cores, return_seconds=True)
        n1 = max(20, sample // 10)
        _, secs1 = r.search_batch(Q[:n1], params["m"], params["K_prime"], params["ef_search"], k=params["k"],
                                  threads=1, return_seconds=True)
        base = {"value": round(len(Qs) / secs, 1), "unit": "queries/s", "cores": cores, "kind": "reference",
                "sample": f"{len(Qs)} of the step's queries, {cores} threads (query-parallel searchRknn)",
                "single_thread": {"value": round(n1 / secs1, 1), "sample": f"{n1} queries, 1 thread"}}
        parity = None
        if plain_ans is not None:
            mism = [i for i in range(len(Qs)) if not np.array_equal(np.asarray(res[i], np.uint64),
                                                                      np.asarray(plain_ans[i], np.uint64))]
            parity = {"queries": len(Qs), "m": params["m"], "K_prime": params["K_prime"],
                      "ef_search": params["ef_search"], "k": params["k"], "threshold": 1.0,
                      "mismatches": len(mism), "first_mismatches": mism[:8],
                      "answers": int(sum(len(x) for x in res))}
            if gt is not None:
                parity["recall_reference"] = round(macro_recall(gt, res), 4)
                parity["recall_gpu_plain"] = round(macro_recall(gt, plain_ans), 4)
        if head_ans is not None and X is not None and kcol is not None:
            # labels are internal ids (the bench inserts in data order)
            qi = np.concatenate([np.full(len(a), i, np.int64) for i, a in enumerate(head_ans)] + [np.zeros(0, np.int64)])
            pi = np.concatenate([np.asarray(a, np.int64) for a in head_ans] + [np.zeros(0, np.int64)])
            d_ref = ref.l2_batch(Qs[qi], X[pi]) if len(qi) else np.zeros(0, np.float32)
            kdp = kcol[pi].astype(np.float32)
            fail = d_ref > kdp
            ulp = np.spacing(kdp).astype(np.float64)
            band = np.abs(d_ref.astype(np.float64) - kdp.astype(np.float64)) <= 16.0 * ulp
            parity = parity or {}
            parity.update({"head_form": head, "head_answers": int(len(qi)),
                           "lowp_false_accepts": int(np.sum(fail & ~band)),
                           "fp64_band_accepts": int(np.sum(fail & band))})
        return base, parity
    finally:
        shutil.rmtree(td, ignore_errors=True)


def cpu_build_baseline(H, torch, dev, dev_sync):
    """The reference's own build (HNSW insertion with the KNN seeds, refineKNNG,
    buildRKNNG; oracle/_ref) on its CPU-runnable case -- 100k x 128, 64 equal
    Gaussians, K_knng=100, ef_construction=400, 10 iterations of S=50 -- with all
    host cores, beside the GPU build of the same points, and the KNN-graph recall
    of both against exact kNN (1000 seeded nodes, each index in its own id order)."""
    from oracle import idx, ref
    if not ref.available():
        return {"kind": "reference", "sample": "oracle/_ref not built"}
    import shutil
    import tempfile
    W1 = WORKLOADS["plain-100k-d128-K100"]
    X1 = mixture(W1["n"], W1["d"], W1["C"], W1["sigma"], W1["seed"], W1["seed"], dirichlet=W1["dirichlet"])
    cores = os.cpu_count() or 1
    out = {"workload": "plain-100k-d128-K100", "kind": "reference", "cores": cores}
    td = tempfile.mkdtemp(prefix="hrnn_build_ref_")
    try:
        with StdoutToStderr():
            r = ref.RefIndex.create(W1["d"], W1["n"], W1["M"], W1["efc"], 100, W1["K"])
            t0 = time.perf_counter()
            r.add_points(X1, threads=cores)
            t1 = time.perf_counter()
            r.refine(W1["iters"], W1["S"], threads=cores)
            t2 = time.perf_counter()
            r.build_rknng()
            t3 = time.perf_counter()
            p = os.path.join(td, "ref.idx")
            r.save(p)
        Xr = idx.read_idx(p).vectors()  # the reference's internal order (parallel insertion)

        class _RefLists:
            def get_knng(self):
                return r.knng(W1["K"])

        out["reference"] = {"hnsw_insert_s": round(t1 - t0, 3), "nndescent_s": round(t2 - t1, 3),
                            "rknng_csr_s": round(t3 - t2, 3), "knng_build_s": round(t3 - t1, 3),
                            "knng_quality": knng_quality(torch, _RefLists(), Xr, W1["K"], dev)}
        del r
        g, b = build_index(H, W1, X1, dev_sync)
        b = {k_: round(v, 3) for k_, v in b.items()}
        b["knng_quality"] = knng_quality(torch, g, X1, W1["K"], dev)
        out["gpu"] = b
        out["speedup_knng_build"] = round(out["reference"]["knng_build_s"] / max(b["knng_build_s"], 1e-9), 1)
        del g
    finally:
        shutil.rmtree(td, ignore_errors=True)
    return out


def run_reference_arm(args, W, h, Q, params, sweep, build):
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (reference compiled from its sources) "
                                                              "not built on this host"}))
        return
    import shutil
    td, p = _save_for_reference(h)
    try:
        r = ref.RefIndex.load(p, W["d"])
        cores = os.cpu_count() or 1
        per_step = W["nq"]

        def sel(v, a, b):  # per-query parameter arrays follow their queries
            return v[a:b] if isinstance(v, np.ndarray) else v

        def run(a, b, secs=False):
            return r.search_batch(Q[a:b], sel(params["m"], a, b), sel(params["K_prime"], a, b),
                                  sel(params["ef_search"], a, b), k=params["k"], threads=cores, return_seconds=secs)

        for i in range(args.warmup):
            run(0, min(200, per_step))
        tot_q, tot_s = 0, 0.0
        for i in range(args.steps):
            a = (i * per_step) % W["nq"]
            res, secs = run(a, a + per_step, True)
            tot_q += len(res)
            tot_s += secs
        v = tot_q / tot_s
        line = {"impl": "reference", "metric": "RkNN queries/s at recall>=0.95 (k=10)", "value": round(v, 1),
                "unit": "queries/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(1e3 * tot_s / args.steps, 3), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Gaussian mixture)",
                "config": {"workload": args.workload, "n": W["n"], "dim": W["d"], "K_knng": W["K"],
                           "queries_per_step": per_step,
                           **{k_: (v_ if not isinstance(v_, np.ndarray) else "per-query, as the GPU arm's")
                              for k_, v_ in params.items()},
                           "index": "the same .idx file (built by the GPU builder; the reference loads it "
                                    "with HRNN(space, path))"},
                "cpu_baseline": {"value": round(v, 1), "unit": "queries/s", "cores": cores, "kind": "reference",
                                 "sample": f"{per_step} queries per step, {cores} threads"},
                "e2e": {"value": round(v, 1), "unit": "queries/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
    finally:
        shutil.rmtree(td, ignore_errors=True)


if __name__ == "__main__":
    main()
