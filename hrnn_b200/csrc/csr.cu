// Reverse KNN graph as a CSR transpose on the device (buildRKNNG, hrnn.h:1869-1935),
// the mutable per-node reverse lists (buildRKNNG_mutable, hrnn.h:1942-1959) and
// the serve-mode kdist matrix (compactForServing, hrnn.h:299-364).
//
// Device algorithm (HBM-bound integer work, no tensor cores):
//   1. histogram of in-degrees with atomics                (reads N*K ids)
//   2. exclusive scan -> u64 offsets, exactly the reference's rknng_offsets_
//   3. scatter (owner << rank_bits) | rank with per-target atomic cursors
//   4. sort every segment by (rank, owner): one warp per segment of <= 1024
//      entries (bitonic network in shared memory), one block per larger segment.
// Step 4 makes the result independent of the scatter order: each segment holds
// exactly the reference's entries, grouped by rank like the reference's, with ties
// in owner order (the reference's std::sort leaves ties in an unspecified order;
// phase B reads whole rank groups, so search results do not depend on it).
// rknng_reference_order() produces the reference's exact byte order on the host
// for saveIndex by applying the same std::sort call to the owner-ordered array.
#include <algorithm>
#include <cstdlib>
#include <cfloat>
#include <vector>

#include "index.hpp"

namespace hrnn {

namespace {

__global__ void k_degree(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ hdr, size_t n,
                         uint32_t K, uint32_t* __restrict__ deg) {
    size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t i = warp; i < n; i += nw) {
        uint32_t c = hdr[i] & 0xFFFFu;
        for (uint32_t j = lane; j < c; j += 32) atomicAdd(&deg[ids[i * K + j]], 1u);
    }
}

template <class E>
__global__ void k_scatter(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ hdr, size_t n,
                          uint32_t K, const uint64_t* __restrict__ off, uint32_t* __restrict__ cursor,
                          E* __restrict__ ent, uint32_t rb) {
    size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t i = warp; i < n; i += nw) {
        uint32_t c = hdr[i] & 0xFFFFu;
        for (uint32_t j = lane; j < c; j += 32) {
            uint32_t nbr = ids[i * K + j];
            uint64_t pos = off[nbr] + atomicAdd(&cursor[nbr], 1u);
            ent[pos] = (E)(((uint64_t)i << rb) | j);
        }
    }
}

// Sort key: rank in the high word, owner in the low word.
template <class E>
__device__ __forceinline__ uint64_t to_key(E e, uint32_t rb) {
    uint64_t v = (uint64_t)e;
    return ((v & ((1ull << rb) - 1)) << 32) | (v >> rb);
}
template <class E>
__device__ __forceinline__ E from_key(uint64_t k, uint32_t rb) {
    return (E)(((k & 0xFFFFFFFFull) << rb) | (k >> 32));
}

constexpr int kWarpSegMax = 1024;
constexpr int kSortWarps = 4;

// Bitonic sort of P (power of two) keys in shared memory by a group of `nthreads`
// threads with thread index t; sync() separates the stages.
template <class Sync>
__device__ void bitonic(uint64_t* s, uint32_t P, uint32_t t, uint32_t nthreads, Sync sync) {
    for (uint32_t k = 2; k <= P; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = t; i < P; i += nthreads) {
                uint32_t p = i ^ j;
                if (p > i) {
                    uint64_t a = s[i], b = s[p];
                    bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        s[i] = b;
                        s[p] = a;
                    }
                }
            }
            sync();
        }
    }
}

template <class E>
__global__ void k_sort_small(const uint64_t* __restrict__ off, size_t n, E* __restrict__ ent, uint32_t rb,
                             uint32_t* __restrict__ big, uint32_t* __restrict__ n_big) {
    __shared__ uint64_t sm[kSortWarps][kWarpSegMax];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    size_t seg = (size_t)blockIdx.x * kSortWarps + w;
    size_t stride = (size_t)gridDim.x * kSortWarps;
    for (; seg < n; seg += stride) {
        uint64_t b = off[seg], e = off[seg + 1];
        uint32_t len = (uint32_t)(e - b);
        if (len <= 1) continue;
        if (len > kWarpSegMax) {
            if (lane == 0) big[atomicAdd(n_big, 1u)] = (uint32_t)seg;
            continue;
        }
        uint32_t P = 32;
        while (P < len) P <<= 1;
        uint64_t* s = sm[w];
        for (uint32_t i = lane; i < P; i += 32) s[i] = i < len ? to_key<E>(ent[b + i], rb) : ~0ull;
        __syncwarp();
        bitonic(s, P, lane, 32, [] { __syncwarp(); });
        for (uint32_t i = lane; i < len; i += 32) ent[b + i] = from_key<E>(s[i], rb);
        __syncwarp();
    }
}

// One block per large segment; keys staged in `tmp` (global) when they do not fit
// the dynamic shared memory.
template <class E>
__global__ void k_sort_big(const uint64_t* __restrict__ off, const uint32_t* __restrict__ big,
                           E* __restrict__ ent, uint32_t rb, uint32_t smem_keys, uint64_t* __restrict__ tmp,
                           size_t tmp_stride) {
    extern __shared__ uint64_t dyn[];
    uint32_t seg = big[blockIdx.x];
    uint64_t b = off[seg], e = off[seg + 1];
    uint32_t len = (uint32_t)(e - b);
    uint32_t P = 32;
    while (P < len) P <<= 1;
    uint64_t* s = (P <= smem_keys) ? dyn : tmp + (size_t)blockIdx.x * tmp_stride;
    for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) s[i] = i < len ? to_key<E>(ent[b + i], rb) : ~0ull;
    __syncthreads();
    bitonic(s, P, threadIdx.x, blockDim.x, [] { __syncthreads(); });
    for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) ent[b + i] = from_key<E>(s[i], rb);
}

__global__ void k_kdist_serve(const uint32_t* __restrict__ hdr, const float* __restrict__ dist, size_t n,
                              uint32_t K, uint32_t mks, float* __restrict__ out) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * mks) return;
    size_t i = t / mks;
    uint32_t j = (uint32_t)(t % mks);
    uint32_t c = hdr[i] & 0xFFFFu;
    out[t] = j < c ? dist[i * K + j] : FLT_MAX;
}

int sm_count(int dev) {
    int v = 148;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v;
}

template <class E>
void build_impl(Index& ix) {
    const size_t n = ix.cur, K = ix.K;
    cudaStream_t s = ix.stream;
    DevMem& deg = ix.scratch[0];
    DevMem& cursor = ix.scratch[1];
    DevMem& big = ix.scratch[2];
    DevMem& tmp = ix.scratch[3];
    deg.ensure((n + 1) * 4);
    cursor.ensure((n + 1) * 4 + 4);
    CUDA_CHECK(cudaMemsetAsync(deg.p, 0, (n + 1) * 4, s));
    CUDA_CHECK(cudaMemsetAsync(cursor.p, 0, (n + 1) * 4 + 4, s));
    int grid = sm_count(ix.device) * 8;
    k_degree<<<grid, 256, 0, s>>>(ix.knn_ids.as<uint32_t>(), ix.knn_hdr.as<uint32_t>(), n, (uint32_t)K,
                                  deg.as<uint32_t>());
    CUDA_LAUNCH_CHECK();
    ix.csr_off.ensure((n + 1) * 8);
    exclusive_scan_u32_to_u64(deg.as<uint32_t>(), ix.csr_off.as<uint64_t>(), n + 1, s, tmp);
    uint64_t total = 0;
    CUDA_CHECK(cudaMemcpyAsync(&total, ix.csr_off.as<uint64_t>() + n, 8, cudaMemcpyDeviceToHost, s));
    CUDA_CHECK(cudaStreamSynchronize(s));
    ix.csr_ent.ensure(std::max<uint64_t>(total, 1) * sizeof(E));
    k_scatter<E><<<grid, 256, 0, s>>>(ix.knn_ids.as<uint32_t>(), ix.knn_hdr.as<uint32_t>(), n, (uint32_t)K,
                                      ix.csr_off.as<uint64_t>(), cursor.as<uint32_t>(), ix.csr_ent.as<E>(),
                                      ix.rank_bits);
    CUDA_LAUNCH_CHECK();
    big.ensure((n + 1) * 4);
    uint32_t* n_big = cursor.as<uint32_t>() + n + 1;  // spare word, zeroed above
    CUDA_CHECK(cudaMemsetAsync(n_big, 0, 4, s));
    size_t blocks = std::min<size_t>((n + kSortWarps - 1) / kSortWarps, (size_t)sm_count(ix.device) * 32);
    k_sort_small<E><<<(unsigned)std::max<size_t>(blocks, 1), kSortWarps * 32, 0, s>>>(
        ix.csr_off.as<uint64_t>(), n, ix.csr_ent.as<E>(), ix.rank_bits, big.as<uint32_t>(), n_big);
    CUDA_LAUNCH_CHECK();
    uint32_t nb = 0;
    CUDA_CHECK(cudaMemcpyAsync(&nb, n_big, 4, cudaMemcpyDeviceToHost, s));
    CUDA_CHECK(cudaStreamSynchronize(s));
    if (nb) {
        // Size the staging area for the largest segment.
        std::vector<uint32_t> bigs(nb);
        CUDA_CHECK(cudaMemcpy(bigs.data(), big.p, nb * 4, cudaMemcpyDeviceToHost));
        std::vector<uint64_t> hoff(n + 1);
        CUDA_CHECK(cudaMemcpy(hoff.data(), ix.csr_off.p, (n + 1) * 8, cudaMemcpyDeviceToHost));
        uint32_t maxlen = 0;
        for (uint32_t sg : bigs) maxlen = std::max<uint32_t>(maxlen, (uint32_t)(hoff[sg + 1] - hoff[sg]));
        uint32_t P = 32;
        while (P < maxlen) P <<= 1;
        const uint32_t smem_keys = 16384;  // 128 KB
        uint64_t* gtmp = nullptr;
        size_t stride = 0;
        if (P > smem_keys) {
            stride = P;
            tmp.ensure((size_t)nb * P * 8 + 64);
            gtmp = tmp.as<uint64_t>();
        }
        size_t smem = (size_t)smem_keys * 8;
        CUDA_CHECK(cudaFuncSetAttribute(k_sort_big<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_sort_big<E><<<nb, 512, smem, s>>>(ix.csr_off.as<uint64_t>(), big.as<uint32_t>(), ix.csr_ent.as<E>(),
                                            ix.rank_bits, smem_keys, gtmp, stride);
        CUDA_LAUNCH_CHECK();
    }
    CUDA_CHECK(cudaStreamSynchronize(s));
    ix.csr_entries = total;
}

template <class E>
void reference_order_impl(size_t n, uint32_t rb, const uint64_t* off, E* ent) {
    // buildRKNNG_fill (hrnn.h:1919-1934): the scatter visits owners in increasing
    // id and each owner's list in rank order, so every segment starts out sorted by
    // the full entry value; the reference then calls std::sort on it with a
    // rank-only comparator.  The same libstdc++ call on the same input gives the
    // same bytes.
    const E mask = (E)((E(1) << rb) - 1);
#pragma omp parallel for schedule(dynamic, 1024)
    for (long long b = 0; b < (long long)n; ++b) {
        E* beg = ent + off[b];
        E* en = ent + off[b + 1];
        std::sort(beg, en);
        std::sort(beg, en, [mask](E a, E c) { return (a & mask) < (c & mask); });
    }
}

}  // namespace

void build_rknng(Index& ix) {
    if (!ix.knng_built) fail(HRNN_ERR_STATE, "buildRKNNG: KNNG not built yet");
    const size_t n = ix.cur;
    uint32_t rb = 0, nb = 0;                              // hrnn.h:1876-1880
    while ((1ull << rb) < ix.K) rb++;
    while ((1ull << nb) < n) nb++;
    if (nb + rb > 64)
        fail(HRNN_ERR_ARG, "buildRKNNG: exceeds 64-bit packing (n=" + std::to_string(n) + " needs " +
                               std::to_string(nb) + " bits, K=" + std::to_string(ix.K) + " needs " +
                               std::to_string(rb) + " bits)");
    ix.rank_bits = rb;
    ix.wide = (nb + rb) > 32;
    // HRNN_RKNNG_WIDE=1 stores 64-bit entries even when 32 bits hold owner and
    // rank: a valid wide CSR (the .idx records the entry width), which lets a
    // small index exercise the path that n * K > 2^32 list slots would take.
    if (const char* fw = std::getenv("HRNN_RKNNG_WIDE"))
        if (fw[0] == '1') ix.wide = true;
    if (ix.wide) build_impl<uint64_t>(ix);
    else build_impl<uint32_t>(ix);
    ix.csr_in_reference_order = false;
    ix.rknng_built = true;
    ix.csr_stale = false;
}

void rknng_reference_order(Index& ix, uint64_t* offsets, void* entries) {
    CUDA_CHECK(cudaStreamSynchronize(ix.stream));
    size_t n = ix.cur;
    size_t eb = ix.wide ? 8 : 4;
    CUDA_CHECK(cudaMemcpy(offsets, ix.csr_off.p, (n + 1) * 8, cudaMemcpyDeviceToHost));
    if (ix.csr_entries)
        CUDA_CHECK(cudaMemcpy(entries, ix.csr_ent.p, ix.csr_entries * eb, cudaMemcpyDeviceToHost));
    if (ix.csr_in_reference_order) return;
    if (ix.wide) reference_order_impl<uint64_t>(n, ix.rank_bits, offsets, static_cast<uint64_t*>(entries));
    else reference_order_impl<uint32_t>(n, ix.rank_bits, offsets, static_cast<uint32_t*>(entries));
}

void compact_for_serving(Index& ix, size_t mks) {
    if (ix.serve_mode) return;                            // hrnn.h:300
    if (ix.K == 0 || !ix.knng_built) fail(HRNN_ERR_STATE, "compactForServing: KNNG not built");
    if (mks == 0 || mks > ix.K) fail(HRNN_ERR_ARG, "compactForServing: max_k_serve must be in [1, K_knng]");
    if (ix.rknng_built) ensure_flat_rknng(ix);
    size_t n = ix.cur;
    ix.kdist_serve.alloc(std::max<size_t>(n * mks, 1) * 4);
    size_t tot = n * mks;
    if (tot)
        k_kdist_serve<<<(unsigned)((tot + 255) / 256), 256, 0, ix.stream>>>(
            ix.knn_hdr.as<uint32_t>(), ix.knn_dist.as<float>(), n, (uint32_t)ix.K, (uint32_t)mks,
            ix.kdist_serve.as<float>());
    CUDA_LAUNCH_CHECK();
    CUDA_CHECK(cudaStreamSynchronize(ix.stream));
    // The KNN slot is dropped from the serving layout, as in the reference.
    ix.knn_ids.release();
    ix.knn_dist.release();
    ix.max_k_serve = mks;
    ix.serve_mode = true;
}

}  // namespace hrnn
