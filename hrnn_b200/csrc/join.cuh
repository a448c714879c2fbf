// Local-join proposals of NNDescent (refineKNNG phase 2, hrnn.h:1823-1853) and the
// launcher of the tensor-core join.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace hrnn {

// One proposal of the local join: `source` may enter `target`'s list at distance d.
struct Prop {
    uint32_t target, source;
    float d;
};

// Join modes of refineKNNG (hrnn_set_join_mode).
constexpr int kJoinExact = 0;   // exact FP32 for every sample pair (CUDA cores)
constexpr int kJoinTensor = 1;  // BF16 Gram screen on the tensor cores, exact FP32 for survivors
constexpr int kJoinAudit = 2;   // the screen, then exact FP32 for every pair, counting screen misses

// Counters of the tensor-core join, accumulated on the device over one chunk.
struct JoinTcCounters {
    unsigned long long survivors;    // pairs the screen passed to exact FP32
    unsigned long long dense_nodes;  // nodes whose survivors overflowed the list (all pairs exact)
    unsigned long long misses;       // audit: proposals the screen would have dropped (must be 0)
    int err;                         // a bounded wait on the tensor-core commit ran out
    int pad;
};

// Whether the tensor-core join supports (dim, sample lists of `cap` entries).
bool join_tc_supported(uint32_t dim, uint32_t cap);

// Tensor-core join of nodes [node0, node1): proposals appended to prop (count in
// *pcount, capped at pcap), pair count added to *njoin.  mode: kJoinTensor or
// kJoinAudit.
void join_tc(const float* vec, uint32_t dim, uint32_t node0, uint32_t node1, uint32_t cap,
             const uint32_t* newl, const uint32_t* newc, const uint32_t* oldl, const uint32_t* oldc,
             const float* thr, Prop* prop, unsigned long long* pcount, unsigned long long pcap,
             unsigned long long* njoin, JoinTcCounters* jc, bool fused, int mode, int nsm, cudaStream_t s);

}  // namespace hrnn
