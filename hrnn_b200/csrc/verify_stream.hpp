// Streaming verification of the INT8 search form (verify_stream.cu).
#pragma once

#include <cstdint>

#include "beam.cuh"
#include "index.hpp"

namespace hrnn {

// Whether the streaming verification applies to this view (dims 96 / 128, the
// reference's 16-lane order, INT8 rows with the INT8 screen on).
bool stream_supported(const DevView& v);
// Sets the verification kernel's launch attributes (call before a stream capture).
void stream_prepare(const DevView& v, bool wide, bool fused);
// Upper bound of the work items for a batch with this many postings and pairs.
size_t stream_max_chunks(uint64_t total_postings, size_t npairs);
// Enqueues the verification of nq queries whose proxies (prox, nq x mmax) have the
// posting prefixes plen; answers in resbuf at res_off, counts in res_count;
// queries with too many acceptances are appended to ovl / *n_ovl for the overflow
// pass.  B must be reserved for (nq, dim, nq * mmax, enough chunks).  grp (may be
// null): only the queries with grp[q] == want are finished (the others' postings
// must have plen 0 -- a batch verified in two groups).
void stream_verify(const DevView& v, bool wide, bool fused, const float* Q, uint32_t nq, uint32_t mmax,
                   const uint32_t* prox, const uint32_t* plen, const uint64_t* res_off, const float* kcol,
                   uint32_t kidx, uint64_t* resbuf, uint32_t* res_count, uint32_t* ovl, uint32_t* n_ovl,
                   SearchCounters* ctr, StreamBufs& B, int nsm, cudaStream_t s, const uint8_t* grp = nullptr,
                   uint8_t want = 0);

}  // namespace hrnn
