// Captured search plans: the batch search (phase A, posting counts, candidate
// verification, result packing) for one fixed batch shape, recorded once as a
// CUDA graph and replayed with no host synchronisation inside.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "index.hpp"

namespace hrnn {

struct SearchPlan {
    Index* ix = nullptr;
    uint64_t generation = 0;       // index generation the plan was captured against
    size_t kernel_nodes = 0;       // kernel launches of one run
    size_t nq = 0, cap = 0;
    uint32_t m_max = 0, ef_max = 0, k = 0;
    float threshold = 1.f;
    // caller-owned device buffers the graph reads and writes
    const float* d_q = nullptr;
    const uint32_t *d_m = nullptr, *d_kp = nullptr, *d_ef = nullptr;
    uint64_t *d_out_off = nullptr, *d_out_lab = nullptr;
    // plan-owned device state (addresses fixed for the graph's lifetime)
    DevMem inputs;    // m and ef clamped to the maxima; clamp flag
    DevMem prox, nprox, plen, qtot, res, kcol, hkey, hcnt, lp, tmp, ctr;
    StreamBufs sb;    // streaming verification (INT8 form)
    // learned budget (captured when enabled at creation): features, MLP
    // activations, frontier distances, decisions and the second search's list,
    // groups, group 1's totals and offsets, stored frontier beams; the second
    // stream the second search runs on, and the events that fork and join it
    DevMem lfeat, lmlp, lproxd, lfb, lgrp, loff, lsaved;
    unsigned long long* budget_levels = nullptr;  // device: queries per budget level of the last run
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~SearchPlan() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (aux) cudaStreamDestroy(aux);
    }
};

// Sizes every buffer for the worst case of the shape (m <= m_max proxies per
// query, every reverse list at most the index's longest), records the search on
// `stream` and instantiates it.  Fails with HRNN_ERR_NOMEM when that bound does
// not fit.  With the learned budget enabled the plan records its search (frontier
// pass, MLP, levels, second search) with the budget's settings at creation.
void plan_create(SearchPlan& p, cudaStream_t stream);
// Launches the graph on `stream`; no host synchronisation.
void plan_run(SearchPlan& p, cudaStream_t stream);
// Waits for `stream`, returns the total result count; *clamped = 1 when some
// query's m or ef_search exceeded the plan's maxima (it ran with the maxima).
uint64_t plan_result(SearchPlan& p, cudaStream_t stream, int* clamped);

}  // namespace hrnn
