// Mutable reverse lists on the device: buildRKNNG_mutable (hrnn.h:1942-1959) and
// their maintenance during insertPointDynamic (hrnn.h:2379-2383: a new point joins
// its neighbours' lists; :2462-2480: an accepted point joins the new point's list
// and leaves the list of the entry it pushed out).
//
// Layout: every element (up to max_elements) owns a slot range of ent[] --
// off[i] (u64), cap[i] slots, len[i] used -- holding the owners (u32) of the KNN
// lists that contain i, in no particular order (the reference's
// std::vector<uint32_t> per node).  Capacities are the in-degree plus slack, and
// K + 32 for elements not inserted yet.
//
// Edits are 64-bit words (list << 32 | owner, bit 31 set for a removal), emitted
// by mutable_register (the lists of newly inserted points) and by the K-smallest
// merge (k_merge_cta: inserted and pushed-out entries).  mutable_apply groups the
// edits by list and lets one warp edit each list in place: removals first (find
// the owner, move the last entry into its slot), then additions.  An edit batch
// holds either the registrations of a batch or the changes of one merge, so no
// pair is both added and removed in one batch.  A list that would overflow its
// capacity, or a removal that finds nothing, sets a flag; the host then lays the
// lists out again from the KNN graph (which is always current) with more slack.
// The lists therefore always equal the transpose of the KNN graph.
#include <algorithm>
#include <cstddef>
#include <cstdio>
#include <vector>

#include "index.hpp"

namespace hrnn {

namespace {

constexpr uint32_t kRemove = 0x80000000u;

__global__ void k_mr_degree(const uint32_t* __restrict__ hdr, const uint32_t* __restrict__ ids, uint32_t n,
                            uint32_t K, uint32_t* __restrict__ deg) {
    const size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t i = warp; i < n; i += nw) {
        const uint32_t c = min(hdr[i] & 0xFFFFu, K);
        for (uint32_t j = lane; j < c; j += 32) atomicAdd(&deg[ids[i * K + j]], 1u);
    }
}

// capacity: in-degree + max(32, in-degree / 2) for the n elements present; K + 32
// (the mean in-degree of a full graph, plus slack) for the ones still to come.
__global__ void k_mr_capacity(const uint32_t* __restrict__ deg, uint32_t n, uint32_t ncap, uint32_t K,
                              uint32_t shift, uint32_t* __restrict__ cap) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncap) return;
    const uint32_t d = i < n ? deg[i] : K;
    cap[i] = (d + max(32u, d >> 1)) << shift;
}

__global__ void k_mr_fill(const uint32_t* __restrict__ hdr, const uint32_t* __restrict__ ids, uint32_t n, uint32_t K,
                          const uint64_t* __restrict__ off, uint32_t* __restrict__ len, uint32_t* __restrict__ ent) {
    const size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t i = warp; i < n; i += nw) {
        const uint32_t c = min(hdr[i] & 0xFFFFu, K);
        for (uint32_t j = lane; j < c; j += 32) {
            const uint32_t y = ids[i * K + j];
            ent[off[y] + atomicAdd(&len[y], 1u)] = (uint32_t)i;
        }
    }
}

// The lists of points x0 .. x0 + nx - 1 as additions (y << 32 | x for y in list(x)).
__global__ void k_mr_register(const uint32_t* __restrict__ hdr, const uint32_t* __restrict__ ids, uint32_t x0,
                              uint32_t nx, uint32_t K, uint64_t* __restrict__ ops,
                              unsigned long long* __restrict__ nops, unsigned long long ops_cap) {
    const size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t t = warp; t < nx; t += nw) {
        const uint32_t x = x0 + (uint32_t)t;
        const uint32_t c = min(hdr[x] & 0xFFFFu, K);
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(nops, (unsigned long long)c);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        for (uint32_t j = lane; j < c; j += 32)
            if (base + j < ops_cap) ops[base + j] = ((uint64_t)ids[(size_t)x * K + j] << 32) | x;
    }
}

__global__ void k_op_count(const uint64_t* __restrict__ ops, unsigned long long nops, uint32_t* __restrict__ cnt) {
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < nops;
         i += (unsigned long long)gridDim.x * blockDim.x)
        atomicAdd(&cnt[(uint32_t)(ops[i] >> 32)], 1u);
}

__global__ void k_op_fill(const uint64_t* __restrict__ ops, unsigned long long nops, const uint64_t* __restrict__ ooff,
                          uint32_t* __restrict__ cur, uint32_t* __restrict__ grouped) {
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < nops;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const uint64_t o = ops[i];
        const uint32_t L = (uint32_t)(o >> 32);
        grouped[ooff[L] + atomicAdd(&cur[L], 1u)] = (uint32_t)o;
    }
}

// One warp per list with edits: removals (find the owner, move the last entry into
// its slot), then additions.  flag[0] counts lists that would overflow, flag[1]
// removals that found nothing.
__global__ void k_mr_apply(uint32_t n, const uint64_t* __restrict__ ooff, const uint32_t* __restrict__ grouped,
                           const uint64_t* __restrict__ off, const uint32_t* __restrict__ cap,
                           uint32_t* __restrict__ len, uint32_t* __restrict__ ent, uint32_t* __restrict__ flag) {
    const size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t L = warp; L < n; L += nw) {
        const uint64_t b = ooff[L], e = ooff[L + 1];
        if (b == e) continue;
        uint32_t* E = ent + off[L];
        uint32_t ln = len[L];
        const uint32_t cp = cap[L];
        for (uint64_t k = b; k < e; ++k) {
            const uint32_t op = grouped[k];
            if (!(op & kRemove)) continue;
            const uint32_t o = op & ~kRemove;
            int pos = -1;
            for (uint32_t j0 = 0; j0 < ln && pos < 0; j0 += 32) {
                const uint32_t j = j0 + lane;
                const uint32_t hit = __ballot_sync(0xFFFFFFFFu, j < ln && E[j] == o);
                if (hit) pos = (int)(j0 + __ffs(hit) - 1);
            }
            if (pos < 0) {
                if (lane == 0) atomicAdd(&flag[1], 1u);
                continue;
            }
            if (lane == 0) E[pos] = E[ln - 1];
            __syncwarp();
            ln--;
        }
        for (uint64_t k0 = b; k0 < e; k0 += 32) {
            const uint64_t k = k0 + lane;
            const uint32_t op = k < e ? grouped[k] : kRemove;
            const bool add = !(op & kRemove);
            const uint32_t ab = __ballot_sync(0xFFFFFFFFu, add);
            const uint32_t r = __popc(ab & ((1u << lane) - 1u));
            if (add && ln + r < cp) E[ln + r] = op;
            if (ln + __popc(ab) > cp) {
                if (lane == 0) atomicAdd(&flag[0], 1u);
                ln = cp;
            } else {
                ln += __popc(ab);
            }
        }
        if (lane == 0) len[L] = ln;
        __syncwarp();
    }
}

int sm_count(int dev) {
    int v = 148;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v;
}

}  // namespace

void mutable_build(Index& ix) {
    MutableLists& M = ix.mr;
    cudaStream_t s = ix.stream;
    const uint32_t n = (uint32_t)ix.cur, ncap = (uint32_t)std::max<size_t>(ix.max_elements, 1), K = (uint32_t)ix.K;
    const int nsm = sm_count(ix.device);
    M.len.ensure(((size_t)ncap + 1) * 4);
    M.cap.ensure(((size_t)ncap + 1) * 4);
    M.off.ensure(((size_t)ncap + 1) * 8);
    CUDA_CHECK(cudaMemsetAsync(M.len.p, 0, ((size_t)ncap + 1) * 4, s));
    k_mr_degree<<<nsm * 8, 256, 0, s>>>(ix.knn_hdr.as<uint32_t>(), ix.knn_ids.as<uint32_t>(), n, K, M.len.as<uint32_t>());
    CUDA_LAUNCH_CHECK();
    k_mr_capacity<<<(ncap + 255) / 256, 256, 0, s>>>(M.len.as<uint32_t>(), n, ncap, K, M.slack_shift,
                                                     M.cap.as<uint32_t>());
    CUDA_LAUNCH_CHECK();
    CUDA_CHECK(cudaMemsetAsync(M.cap.as<uint32_t>() + ncap, 0, 4, s));
    exclusive_scan_u32_to_u64(M.cap.as<uint32_t>(), M.off.as<uint64_t>(), (size_t)ncap + 1, s, M.tmp);
    uint64_t total = 0;
    CUDA_CHECK(cudaMemcpyAsync(&total, M.off.as<uint64_t>() + ncap, 8, cudaMemcpyDeviceToHost, s));
    CUDA_CHECK(cudaStreamSynchronize(s));
    M.ent.ensure(std::max<uint64_t>(total, 1) * 4);
    CUDA_CHECK(cudaMemsetAsync(M.len.p, 0, ((size_t)ncap + 1) * 4, s));
    k_mr_fill<<<nsm * 8, 256, 0, s>>>(ix.knn_hdr.as<uint32_t>(), ix.knn_ids.as<uint32_t>(), n, K,
                                      M.off.as<uint64_t>(), M.len.as<uint32_t>(), M.ent.as<uint32_t>());
    CUDA_LAUNCH_CHECK();
    M.ctl.ensure(64);
    CUDA_CHECK(cudaMemsetAsync(M.ctl.p, 0, 64, s));
    M.valid = true;
    M.rebuilds++;
}

void mutable_ops_reserve(Index& ix, unsigned long long cap) {
    MutableLists& M = ix.mr;
    if (M.ops_cap < cap) {
        M.ops.alloc(cap * 8);
        M.ops_cap = cap;
    }
    M.ctl.ensure(64);
}

void mutable_register(Index& ix, uint32_t x0, uint32_t nx) {
    MutableLists& M = ix.mr;
    if (!M.valid || nx == 0) return;
    mutable_ops_reserve(ix, (unsigned long long)nx * std::max<size_t>(ix.K, 1));
    cudaStream_t s = ix.stream;
    unsigned long long* nops = M.ctl.as<unsigned long long>();
    CUDA_CHECK(cudaMemsetAsync(nops, 0, 8, s));
    const int nsm = sm_count(ix.device);
    k_mr_register<<<nsm * 8, 256, 0, s>>>(ix.knn_hdr.as<uint32_t>(), ix.knn_ids.as<uint32_t>(), x0, nx,
                                          (uint32_t)ix.K, M.ops.as<uint64_t>(), nops, M.ops_cap);
    CUDA_LAUNCH_CHECK();
    mutable_apply(ix);
}

void mutable_apply(Index& ix) {
    MutableLists& M = ix.mr;
    if (!M.valid) return;
    cudaStream_t s = ix.stream;
    unsigned long long nops = 0;
    CUDA_CHECK(cudaMemcpyAsync(&nops, M.ctl.p, 8, cudaMemcpyDeviceToHost, s));
    CUDA_CHECK(cudaStreamSynchronize(s));
    const uint32_t n = (uint32_t)ix.cur;
    if (nops > M.ops_cap) {  // edits lost: lay the lists out again from the graph
        mutable_build(ix);
        return;
    }
    if (nops == 0) return;
    const int nsm = sm_count(ix.device);
    M.ocnt.ensure(((size_t)n + 1) * 4);
    M.ocur.ensure(((size_t)n + 1) * 4);
    M.ooff.ensure(((size_t)n + 1) * 8);
    M.grouped.ensure(nops * 4);
    CUDA_CHECK(cudaMemsetAsync(M.ocnt.p, 0, ((size_t)n + 1) * 4, s));
    CUDA_CHECK(cudaMemsetAsync(M.ocur.p, 0, ((size_t)n + 1) * 4, s));
    const unsigned g = (unsigned)std::min<unsigned long long>((nops + 255) / 256, (unsigned long long)nsm * 32);
    k_op_count<<<g, 256, 0, s>>>(M.ops.as<uint64_t>(), nops, M.ocnt.as<uint32_t>());
    CUDA_LAUNCH_CHECK();
    exclusive_scan_u32_to_u64(M.ocnt.as<uint32_t>(), M.ooff.as<uint64_t>(), (size_t)n + 1, s, M.tmp);
    k_op_fill<<<g, 256, 0, s>>>(M.ops.as<uint64_t>(), nops, M.ooff.as<uint64_t>(), M.ocur.as<uint32_t>(),
                                M.grouped.as<uint32_t>());
    CUDA_LAUNCH_CHECK();
    uint32_t* flag = (uint32_t*)(M.ctl.as<char>() + 16);
    CUDA_CHECK(cudaMemsetAsync(flag, 0, 8, s));
    k_mr_apply<<<nsm * 16, 256, 0, s>>>(n, M.ooff.as<uint64_t>(), M.grouped.as<uint32_t>(), M.off.as<uint64_t>(),
                                        M.cap.as<uint32_t>(), M.len.as<uint32_t>(), M.ent.as<uint32_t>(), flag);
    CUDA_LAUNCH_CHECK();
    uint32_t hf[2] = {0, 0};
    CUDA_CHECK(cudaMemcpyAsync(hf, flag, 8, cudaMemcpyDeviceToHost, s));
    CUDA_CHECK(cudaMemsetAsync(M.ctl.p, 0, 8, s));
    CUDA_CHECK(cudaStreamSynchronize(s));
    M.applied += nops;
    if (hf[0] || hf[1]) {  // a list outgrew its slots (or an edit was inconsistent)
        if (hf[0]) M.slack_shift = std::min<uint32_t>(M.slack_shift + 1, 4);
        mutable_build(ix);
    }
}

void mutable_get(Index& ix, uint64_t* lens, uint32_t* flat) {
    MutableLists& M = ix.mr;
    if (!M.valid) fail(HRNN_ERR_STATE, "mutable reverse lists not built (buildRKNNG_mutable)");
    const size_t n = ix.cur;
    if (n == 0) return;
    std::vector<uint32_t> ln(n);
    std::vector<uint64_t> of(n + 1);
    CUDA_CHECK(cudaStreamSynchronize(ix.stream));
    CUDA_CHECK(cudaMemcpy(ln.data(), M.len.p, n * 4, cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(of.data(), M.off.p, (n + 1) * 8, cudaMemcpyDeviceToHost));
    if (lens)
        for (size_t i = 0; i < n; ++i) lens[i] = ln[i];
    if (flat) {
        std::vector<uint32_t> all(of[n]);
        if (of[n]) CUDA_CHECK(cudaMemcpy(all.data(), M.ent.p, of[n] * 4, cudaMemcpyDeviceToHost));
        size_t pos = 0;
        for (size_t i = 0; i < n; ++i) {
            std::copy(all.begin() + (ptrdiff_t)of[i], all.begin() + (ptrdiff_t)(of[i] + ln[i]), flat + pos);
            pos += ln[i];
        }
    }
}

}  // namespace hrnn
