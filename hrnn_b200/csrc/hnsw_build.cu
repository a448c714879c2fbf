// Batched HNSW insertion on the device: the addPoint loop of hrnn_build
// (src/hrnn_build.cpp:75-88; addPoint hrnn.h:1378-1517) with the KNN-graph seed
// of hrnn.h:1479-1501.
//
// Points are inserted in batches that grow with the index (1/24 of the current
// size, at most 16384 points).  For every point of a batch one warp runs, against
// the graph as it was at the start of the batch:
//   - the greedy descent from the entry point down to the point's level + 1;
//   - per level l <= min(level, maxlevel): the ef_construction beam search of
//     that layer (beam.cuh), the KNN-graph seed at level 0 (the beam, ascending,
//     self excluded, at most K entries), and the neighbour heuristic
//     getNeighborsByHeuristic2 (hrnn.h:619-659) choosing at most M links, written
//     in the reference's order (farthest first, hrnn.h:695-699) -- the nearest
//     link is the entry point of the next level (hrnn.h:700);
//   - one reverse-link request (target list, new point, distance) per link.
// Then k_link_update applies all requests of the batch, one warp per target
// list: new points are appended while the list has room, otherwise the union of
// the list and the new points is pruned with the same heuristic to maxM0 (level
// 0) or maxM links (mutuallyConnectNewElement, hrnn.h:729-797).
//
// Levels come from the reference's generator in insertion order
// (getRandomLevel, hrnn.h:383-387; std::default_random_engine seeded with
// random_seed).  Points of one batch do not see each other while searching; the
// graph therefore differs from a sequential build (as the reference's own
// multi-threaded build does), while every stored distance is the exact FP32 value
// of the reference's L2 order.
#include <algorithm>
#include <cstdlib>
#include <cfloat>
#include <cmath>
#include <random>
#include <vector>

#include "beam.cuh"
#include "index.hpp"

namespace hrnn {

DevView make_view(Index& ix);

namespace {

struct LinkReq {
    uint32_t key;     // target list: node id for level 0, cap + upper block index above
    uint32_t target;  // node that owns the list
    uint32_t src;     // new point
    float d;          // L2(new point, target)
};

constexpr uint32_t kMaxSel = 64;      // M of the heuristic (maxM0 for reverse pruning)
constexpr uint32_t kGroupMax = 1024;  // new links applied to one list per batch

// Heuristic of hrnn.h:619-659 on a candidate list sorted by distance to the base
// point: keep a candidate unless a kept one is closer to it than the base is.
// cand ids/dists in shared memory; cq = scratch for one vector; sel outputs.
// Returns the number kept (all candidates when fewer than M).
template <bool FUSED>
__device__ uint32_t heuristic(const DevView& v, const uint32_t* cid, const float* cdist, uint32_t nc, uint32_t M,
                              float* cq, uint32_t* sel_id, float* sel_d, float* tmpd) {
    const int lane = threadIdx.x & 31;
    if (nc < M) {
        for (uint32_t i = lane; i < nc; i += 32) {
            sel_id[i] = cid[i];
            sel_d[i] = cdist[i];
        }
        __syncwarp();
        return nc;
    }
    uint32_t ns = 0;
    for (uint32_t i = 0; i < nc && ns < M; ++i) {
        const uint32_t c = cid[i];
        const float dq = cdist[i];
        bool good = true;
        if (ns) {
            for (uint32_t e = lane; e < v.dim; e += 32) cq[e] = v.vec[(size_t)c * v.dim + e];
            __syncwarp();
            for (uint32_t b = 0; b < ns; b += 32) {
                uint32_t cnt = min(32u, ns - b);
                warp_l2_list<FUSED>(v, cq, sel_id + b, cnt, tmpd);
                bool bad = (uint32_t)lane < cnt && tmpd[lane] < dq;
                if (__any_sync(0xFFFFFFFFu, bad)) {
                    good = false;
                    break;
                }
            }
        }
        if (good) {
            if (lane == 0) {
                sel_id[ns] = c;
                sel_d[ns] = dq;
            }
            ns++;
        }
        __syncwarp();
    }
    return ns;
}

template <bool FUSED>
__global__ void __launch_bounds__(128) k_build_batch(DevView v, uint32_t b0, uint32_t b1, uint32_t ep, int maxlevel,
                                                     uint32_t efc, uint32_t vc, uint32_t M, uint32_t cap,
                                                     const int32_t* __restrict__ levels, uint32_t K,
                                                     uint32_t* __restrict__ knn_hdr, uint32_t* __restrict__ knn_ids,
                                                     float* __restrict__ knn_dist, uint32_t* __restrict__ adj0,
                                                     uint32_t* __restrict__ upper, LinkReq* __restrict__ reqs,
                                                     unsigned long long* __restrict__ nreq) {
    extern __shared__ char smem_raw[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const size_t per_warp = warp_smem_bytes(v.dim, efc, vc) + (size_t)v.dim * 4 + kMaxSel * 12 + 128;
    char* base = smem_raw + (size_t)w * per_warp;
    WarpSmem s = carve(base, v.dim, efc, vc);
    float* cq = (float*)(base + warp_smem_bytes(v.dim, efc, vc));
    uint32_t* sel_id = (uint32_t*)(cq + v.dim);
    float* sel_d = (float*)(sel_id + kMaxSel);
    float* tmpd = sel_d + kMaxSel;
    unsigned long long c_dist = 0, c_exp = 0;
    for (uint32_t p = b0 + blockIdx.x * wpb + w; p < b1; p += gridDim.x * wpb) {
        for (uint32_t i = lane; i < v.dim; i += 32) s.q[i] = v.vec[(size_t)p * v.dim + i];
        __syncwarp();
        const int L = levels[p];
        uint32_t cur = ep;
        float curd = warp_l2_one<FUSED>(v, s.q, cur);
        if (L < maxlevel) greedy_descent<FUSED ? 1 : 0>(v, s, maxlevel, L, cur, curd, c_dist);  // hrnn.h:1438-1464
        for (int level = min(L, maxlevel); level >= 0; --level) {
            uint32_t tsize = beam_search<FUSED ? 1 : 0>(v, s, cur, curd, efc, level, vc, c_dist, c_exp);
            for (uint32_t i = lane; i < tsize; i += 32) s.ti[i] &= kIdMask;
            __syncwarp();
            if (level == 0 && K > 0) {  // KNN-graph seed, hrnn.h:1479-1501
                uint32_t cnt = min(tsize, K);
                for (uint32_t i = lane; i < cnt; i += 32) {
                    knn_ids[(size_t)p * K + i] = s.ti[i];
                    knn_dist[(size_t)p * K + i] = s.td[i];
                }
                if (lane == 0) knn_hdr[p] = cnt;
            }
            uint32_t ns = heuristic<FUSED>(v, s.ti, s.td, tsize, M, cq, sel_id, sel_d, tmpd);
            uint32_t* own = level == 0 ? adj0 + (size_t)p * v.W0 : upper + v.upper_off[p] + (size_t)(level - 1) * v.WU;
            for (uint32_t i = lane; i < ns; i += 32) own[1 + i] = sel_id[ns - 1 - i];  // farthest first
            if (lane == 0) own[0] = ns;
            // reverse-link requests
            unsigned long long rb = 0;
            if (lane == 0) rb = atomicAdd(nreq, (unsigned long long)ns);
            rb = __shfl_sync(0xFFFFFFFFu, rb, 0);
            for (uint32_t i = lane; i < ns; i += 32) {
                uint32_t t = sel_id[i];
                uint32_t key = level == 0 ? t : cap + (uint32_t)(v.upper_off[t] / v.WU) + (uint32_t)(level - 1);
                reqs[rb + i] = LinkReq{key, t, p, sel_d[i]};
            }
            cur = sel_id[0];
            curd = sel_d[0];
            __syncwarp();
        }
    }
}

__global__ void k_req_count(const LinkReq* __restrict__ reqs, unsigned long long nr, uint32_t* __restrict__ cnt,
                            uint32_t* __restrict__ active, uint32_t* __restrict__ nactive,
                            uint32_t* __restrict__ slot_of) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nr; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t key = reqs[i].key;
        if (atomicAdd(&cnt[key], 1u) == 0) {
            uint32_t a = atomicAdd(nactive, 1u);
            active[a] = key;
            slot_of[key] = a;
        }
    }
}

__global__ void k_req_gather_counts(const uint32_t* __restrict__ active, uint32_t na, const uint32_t* __restrict__ cnt,
                                    uint32_t* __restrict__ acnt) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < na) acnt[i] = cnt[active[i]];
    if (i == na) acnt[i] = 0;
}

__global__ void k_req_scatter(const LinkReq* __restrict__ reqs, unsigned long long nr,
                              const uint32_t* __restrict__ slot_of, const uint64_t* __restrict__ aoff,
                              uint32_t* __restrict__ acur, LinkReq* __restrict__ grouped) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nr; i += (size_t)gridDim.x * blockDim.x) {
        LinkReq r = reqs[i];
        uint32_t a = slot_of[r.key];
        grouped[aoff[a] + atomicAdd(&acur[a], 1u)] = r;
    }
}

// Shared memory of one k_link_update warp.
__host__ __device__ inline size_t link_warp_bytes(uint32_t dim) {
    const size_t CMAX = kGroupMax + kMaxSel;
    return (size_t)dim * 8 + CMAX * 8 + CMAX * 8 + kMaxSel * 12 + 32 * 4 + 256;
}

// One warp per target list with new links (mutuallyConnectNewElement, hrnn.h:729-797).
template <bool FUSED>
__global__ void __launch_bounds__(128) k_link_update(DevView v, const uint32_t* __restrict__ active, uint32_t na,
                                                     const uint64_t* __restrict__ aoff, const LinkReq* __restrict__ grp,
                                                     uint32_t cap, uint32_t maxM0, uint32_t maxM,
                                                     uint32_t* __restrict__ adj0, uint32_t* __restrict__ upper,
                                                     uint32_t* __restrict__ cnt_reset) {
    extern __shared__ char smem_raw[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const uint32_t CMAX = kGroupMax + kMaxSel;
    char* base = smem_raw + (size_t)w * link_warp_bytes(v.dim);
    float* sq = (float*)base;                          // target vector
    float* cq = sq + v.dim;                            // candidate vector (heuristic)
    uint64_t* keys = (uint64_t*)(cq + v.dim);          // (d, id) sort keys
    uint32_t* cid = (uint32_t*)(keys + CMAX);          // candidates, ascending
    float* cd = (float*)(cid + CMAX);
    uint32_t* sel_id = (uint32_t*)(cd + CMAX);
    float* sel_d = (float*)(sel_id + kMaxSel);
    uint32_t* eid = (uint32_t*)(sel_d + kMaxSel);      // existing links
    float* tmpd = (float*)(eid + kMaxSel);
    for (uint32_t g = blockIdx.x * wpb + w; g < na; g += gridDim.x * wpb) {
        const uint32_t key = active[g];
        const uint64_t b = aoff[g];
        const uint64_t ng = aoff[g + 1] - b;
        const uint32_t nn = ng < kGroupMax ? (uint32_t)ng : kGroupMax;
        const uint32_t t = grp[b].target;
        const bool lvl0 = key < cap;
        uint32_t* list = lvl0 ? adj0 + (size_t)t * v.W0 : upper + (size_t)(key - cap) * v.WU;
        const uint32_t Mcur = lvl0 ? maxM0 : maxM;
        const uint32_t c0 = list[0] & 0xFFFFu;
        // new links sorted by (distance, id)
        uint32_t P = 32;
        while (P < nn) P <<= 1;
        for (uint32_t x = lane; x < P; x += 32) {
            uint64_t k = ~0ull;
            if (x < nn) {
                LinkReq r = grp[b + x];
                k = ((uint64_t)__float_as_uint(r.d) << 32) | r.src;
            }
            keys[x] = k;
        }
        for (uint32_t kk = 2; kk <= P; kk <<= 1)
            for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
                __syncwarp();
                for (uint32_t x = lane; x < P; x += 32) {
                    uint32_t y = x ^ j;
                    if (y > x) {
                        uint64_t a = keys[x], c = keys[y];
                        if ((a > c) == ((x & kk) == 0)) {
                            keys[x] = c;
                            keys[y] = a;
                        }
                    }
                }
            }
        __syncwarp();
        if (c0 + nn <= Mcur) {  // room for all: append (hrnn.h:759-761)
            for (uint32_t x = lane; x < nn; x += 32) list[1 + c0 + x] = (uint32_t)keys[x];
            __syncwarp();
            if (lane == 0) list[0] = (list[0] & 0xFFFF0000u) | (c0 + nn);
            __syncwarp();
            continue;
        }
        // candidates: the new links and the existing ones with their distance to the
        // target (hrnn.h:766-774), then ordered by (distance, id)
        for (uint32_t e = lane; e < v.dim; e += 32) sq[e] = v.vec[(size_t)t * v.dim + e];
        for (uint32_t x = lane; x < c0; x += 32) eid[x] = list[1 + x];
        for (uint32_t x = lane; x < nn; x += 32) {
            cid[x] = (uint32_t)keys[x];
            cd[x] = __uint_as_float((uint32_t)(keys[x] >> 32));
        }
        __syncwarp();
        for (uint32_t bb = 0; bb < c0; bb += 32) {
            uint32_t cnt = min(32u, c0 - bb);
            warp_l2_list<FUSED>(v, sq, eid + bb, cnt, tmpd);
            if ((uint32_t)lane < cnt) {
                cid[nn + bb + lane] = eid[bb + lane];
                cd[nn + bb + lane] = tmpd[lane];
            }
            __syncwarp();
        }
        const uint32_t total = c0 + nn;
        for (uint32_t x = lane; x < total; x += 32) {
            float dx = cd[x];
            uint32_t ix_ = cid[x], r = 0;
            for (uint32_t y = 0; y < total; ++y) {
                float dy = cd[y];
                r += (dy < dx) || (dy == dx && cid[y] < ix_);
            }
            keys[r] = ((uint64_t)__float_as_uint(dx) << 32) | ix_;
        }
        __syncwarp();
        for (uint32_t x = lane; x < total; x += 32) {
            cid[x] = (uint32_t)keys[x];
            cd[x] = __uint_as_float((uint32_t)(keys[x] >> 32));
        }
        __syncwarp();
        uint32_t ns = heuristic<FUSED>(v, cid, cd, total, Mcur, cq, sel_id, sel_d, tmpd);
        for (uint32_t i = lane; i < ns; i += 32) list[1 + i] = sel_id[ns - 1 - i];
        __syncwarp();
        if (lane == 0) list[0] = (list[0] & 0xFFFF0000u) | ns;
        __syncwarp();
    }
    // reset the per-key counters of this batch
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < na; g += gridDim.x * blockDim.x) cnt_reset[active[g]] = 0;
}

int nsm_of(int dev) {
    int v = 148;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v;
}

}  // namespace

void add_points(Index& ix, const float* data, const uint64_t* labels, size_t n_add) {
    if (n_add == 0) return;
    if (ix.serve_mode) fail(HRNN_ERR_STATE, "addPoint: index is in serve mode");
    if (ix.cur + n_add > ix.max_elements)
        fail(HRNN_ERR_LIMIT, "The number of elements exceeds the specified limit");   // hrnn.h:1402-1404
    if (ix.maxM0 > kMaxSel || ix.M > kMaxSel) fail(HRNN_ERR_ARG, "addPoint: M above 32 is not supported");
    const size_t b_start = ix.cur, end = ix.cur + n_add, dim = ix.dim;
    std::vector<uint64_t> lab(n_add);
    for (size_t i = 0; i < n_add; ++i) {
        lab[i] = labels ? labels[i] : (uint64_t)(b_start + i);
        if (!ix.label_lookup.emplace(lab[i], (uint32_t)(b_start + i)).second) {
            for (size_t j = 0; j < i; ++j) ix.label_lookup.erase(lab[j]);
            fail(HRNN_ERR_ARG, "addPoint: label already present (updates are not supported)");
        }
    }
    cudaStream_t s = ix.stream;
    CUDA_CHECK(cudaMemcpyAsync(ix.vec.as<float>() + b_start * dim, data, n_add * dim * 4, cudaMemcpyHostToDevice, s));
    CUDA_CHECK(cudaMemcpyAsync(ix.labels.as<uint64_t>() + b_start, lab.data(), n_add * 8, cudaMemcpyHostToDevice, s));
    // Levels in insertion order from the reference's generator (hrnn.h:383-387).
    std::uniform_real_distribution<double> U(0.0, 1.0);
    for (size_t i = b_start; i < end; ++i) {
        int lv = (int)(-std::log(U(ix.level_generator)) * ix.mult);
        ix.levels[i] = lv;
        ix.upper_off[i] = ix.upper.size();
        if (lv > 0) ix.upper.resize(ix.upper.size() + (size_t)lv * (1 + ix.maxM), 0u);
    }
    ix.upper_dirty = true;
    ix.sync_upper_to_device();
    DevMem d_levels;
    d_levels.alloc(end * 4);
    CUDA_CHECK(cudaMemcpyAsync(d_levels.p, ix.levels.data(), end * 4, cudaMemcpyHostToDevice, s));
    // Scratch for link requests and their grouping.
    const uint32_t cap = (uint32_t)ix.max_elements;
    const size_t keyspace = cap + ix.upper.size() / (1 + ix.maxM) + 1;
    const size_t max_batch = 16384;
    size_t maxreq = max_batch * ix.M * 8 + 1024;
    DevMem reqs, grouped, kcnt, slot_of, active, acnt, aoff, acur, ctr, tmp;
    reqs.alloc(maxreq * sizeof(LinkReq));
    grouped.alloc(maxreq * sizeof(LinkReq));
    kcnt.alloc(keyspace * 4);
    slot_of.alloc(keyspace * 4);
    active.alloc(maxreq * 4);
    acnt.alloc((maxreq + 1) * 4);
    aoff.alloc((maxreq + 1) * 8);
    acur.alloc((maxreq + 1) * 4);
    ctr.alloc(64);
    CUDA_CHECK(cudaMemsetAsync(kcnt.p, 0, kcnt.bytes, s));
    const int nsm = nsm_of(ix.device);
    const bool fused = (ix.order.fused & 1) != 0;
    const uint32_t efc = (uint32_t)((ix.ef_construction + 31) & ~(size_t)31);
    // Visited-cache slots per warp (lossy: a miss only re-scores a node, so the
    // graph does not depend on it); HRNN_BUILD_VC overrides, for measurements.
    uint32_t vc = 2048;
    if (const char* e = std::getenv("HRNN_BUILD_VC")) {
        const unsigned long v = std::strtoul(e, nullptr, 10);
        if (v >= 256 && v <= 8192 && (v & (v - 1)) == 0) vc = (uint32_t)v;
    }
    const size_t per_warp_b = warp_smem_bytes((uint32_t)dim, efc, vc) + dim * 4 + kMaxSel * 12 + 128;
    const int wpb = (int)std::max<size_t>(1, std::min<size_t>(4, (200 * 1024) / per_warp_b));
    const size_t smem_b = per_warp_b * wpb;
    const size_t smem_l = link_warp_bytes((uint32_t)dim) * 4;
    if (smem_b > 227 * 1024 || smem_l > 227 * 1024) fail(HRNN_ERR_ARG, "addPoint: dim/ef_construction too large");
    auto kb = fused ? k_build_batch<true> : k_build_batch<false>;
    auto kl = fused ? k_link_update<true> : k_link_update<false>;
    CUDA_CHECK(cudaFuncSetAttribute(kb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_b));
    CUDA_CHECK(cudaFuncSetAttribute(kl, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_l));
    size_t pos = b_start;
    if (ix.cur == 0 && ix.enterpoint == kInvalid) {  // first element (hrnn.h:1505-1509)
        ix.enterpoint = 0;
        ix.maxlevel = ix.levels[0];
        pos = 1;
    }
    unsigned long long* d_nreq = ctr.as<unsigned long long>();
    uint32_t* d_nact = (uint32_t*)(d_nreq + 1);
    while (pos < end) {
        size_t batch = std::max<size_t>(1, std::min<size_t>(pos / 24, max_batch));
        size_t b1 = std::min(end, pos + batch);
        ix.cur = b1;  // view covers the batch (vectors); the graph does not reach it yet
        DevView v = make_view(ix);
        CUDA_CHECK(cudaMemsetAsync(ctr.p, 0, 64, s));
        unsigned grid = (unsigned)std::min<size_t>((b1 - pos + wpb - 1) / wpb, (size_t)nsm * 8);
        kb<<<grid, wpb * 32, smem_b, s>>>(v, (uint32_t)pos, (uint32_t)b1, ix.enterpoint, ix.maxlevel, efc, vc,
                                          (uint32_t)ix.M, cap, d_levels.as<int32_t>(), (uint32_t)ix.K,
                                          ix.knn_hdr.as<uint32_t>(), ix.knn_ids.as<uint32_t>(),
                                          ix.knn_dist.as<float>(), ix.adj0.as<uint32_t>(), ix.d_upper.as<uint32_t>(),
                                          reqs.as<LinkReq>(), d_nreq);
        CUDA_LAUNCH_CHECK();
        unsigned long long nr = 0;
        CUDA_CHECK(cudaMemcpyAsync(&nr, d_nreq, 8, cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaStreamSynchronize(s));
        if (nr > maxreq) fail(HRNN_ERR_STATE, "addPoint: link request buffer overflow");
        if (nr) {
            unsigned g = (unsigned)std::min<unsigned long long>((nr + 255) / 256, (unsigned long long)nsm * 16);
            k_req_count<<<g, 256, 0, s>>>(reqs.as<LinkReq>(), nr, kcnt.as<uint32_t>(), active.as<uint32_t>(), d_nact,
                                          slot_of.as<uint32_t>());
            CUDA_LAUNCH_CHECK();
            uint32_t na = 0;
            CUDA_CHECK(cudaMemcpyAsync(&na, d_nact, 4, cudaMemcpyDeviceToHost, s));
            CUDA_CHECK(cudaStreamSynchronize(s));
            k_req_gather_counts<<<(na + 256) / 256, 256, 0, s>>>(active.as<uint32_t>(), na, kcnt.as<uint32_t>(),
                                                                acnt.as<uint32_t>());
            CUDA_LAUNCH_CHECK();
            exclusive_scan_u32_to_u64(acnt.as<uint32_t>(), aoff.as<uint64_t>(), (size_t)na + 1, s, tmp);
            CUDA_CHECK(cudaMemsetAsync(acur.p, 0, ((size_t)na + 1) * 4, s));
            k_req_scatter<<<g, 256, 0, s>>>(reqs.as<LinkReq>(), nr, slot_of.as<uint32_t>(), aoff.as<uint64_t>(),
                                            acur.as<uint32_t>(), grouped.as<LinkReq>());
            CUDA_LAUNCH_CHECK();
            unsigned gl = (unsigned)std::min<size_t>(((size_t)na + 3) / 4, (size_t)nsm * 8);
            kl<<<std::max(1u, gl), 128, smem_l, s>>>(v, active.as<uint32_t>(), na, aoff.as<uint64_t>(),
                                                     grouped.as<LinkReq>(), cap, (uint32_t)ix.maxM0, (uint32_t)ix.maxM,
                                                     ix.adj0.as<uint32_t>(), ix.d_upper.as<uint32_t>(),
                                                     kcnt.as<uint32_t>());
            CUDA_LAUNCH_CHECK();
        }
        // entry point: first point of the batch with the highest level above maxlevel
        for (size_t i = pos; i < b1; ++i)
            if (ix.levels[i] > ix.maxlevel) {
                ix.maxlevel = ix.levels[i];
                ix.enterpoint = (uint32_t)i;
            }
        pos = b1;
    }
    CUDA_CHECK(cudaStreamSynchronize(s));
    ix.cur = end;
    ix.bf16_valid = false;  // the BF16 / INT8 copies are rebuilt on the next search that uses them
    ix.i8_valid = false;
    // The reverse lists no longer cover every point: searches need buildRKNNG first
    // (the reference leaves its flag set and would read past its offsets array).
    ix.rknng_built = false;
    // The device copy of the upper layers is now authoritative; mirror it back.
    if (!ix.upper.empty())
        CUDA_CHECK(cudaMemcpy(ix.upper.data(), ix.d_upper.p, ix.upper.size() * 4, cudaMemcpyDeviceToHost));
    ix.upper_dirty = false;
}

}  // namespace hrnn
