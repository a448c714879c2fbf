// NNDescent refinement of the KNN graph on the device (refineKNNG, hrnn.h:1725-1862).
//
// One iteration of the reference, run on one thread, ends with every list equal to
// the K smallest distinct (distance, id) pairs of (its list at the start of the
// iteration) U (all proposals the local join makes for it): try_update_knng_nnd
// (hrnn.h:1660-1722) inserts with early rejection against the current farthest
// entry and evicts the farthest, and a pair rejected or evicted once can never
// re-enter.  The join's pairs depend only on the sample lists fixed in phase 1.
// So the device computes the same iteration in bulk:
//
//   phase 1  k_sample_count / k_sample_fill / k_sample_rev:
//            first S new and first S old entries by rank (hrnn.h:1764-1805), new
//            flags cleared; reverse samples capped at R keep the R smallest owner
//            ids -- the ones a single thread visiting owners in increasing id
//            pushes first (hrnn.h:1781-1790, 1797-1804); lists merged (:1813-1819).
//   phase 2  nodes processed in chunks.  k_join computes every new x new (i<j) and
//            new x old pair of a node in exact FP32 (the reference's order) and
//            emits (target, source, d) proposals that can still enter the target's
//            list (d below its current farthest when the list is full);
//            k_bucket_* group them by target; k_merge sorts each target's
//            proposals (bitonic, shared memory), drops duplicates and ids already
//            listed, and merges them into the sorted list keeping K, marking the
//            inserted entries new.  Chunking changes nothing in the result (the
//            outcome is order-independent) but bounds the proposal buffer: lists
//            fill during the first chunk, after which the threshold filters.
//
// Equal distances between different ids are the one place where the bulk merge and
// the sequential insertion can order entries differently.
#include <algorithm>
#include <cfloat>
#include <cstdio>
#include <vector>

#include "index.hpp"

namespace hrnn {

namespace {

constexpr uint32_t kMaxK = 2048;

__device__ __forceinline__ uint32_t lanemask_lt_() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ float worst_of(const uint32_t* hdr, const float* dist, uint32_t K, uint32_t u) {
    uint32_t c = hdr[u] & 0xFFFFu;
    return c >= K ? dist[(size_t)u * K + c - 1] : FLT_MAX;
}

// ---- phase 1 -----------------------------------------------------------------

__global__ void k_init_flags(const uint32_t* __restrict__ hdr, uint32_t n, uint32_t K, uint8_t* __restrict__ f) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < (size_t)n * K) f[t] = (uint32_t)(t % K) < (hdr[t / K] & 0xFFFFu);
}

// Counts reverse-sample candidates per (target, type) segment: seg = 2*nbr + (old?1:0).
__global__ void k_sample_count(const uint32_t* __restrict__ ids, const float* __restrict__ dist,
                               const uint32_t* __restrict__ hdr, const uint8_t* __restrict__ isnew, uint32_t n,
                               uint32_t K, uint32_t* __restrict__ rcount) {
    size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t i = warp; i < n; i += nw) {
        uint32_t c = hdr[i] & 0xFFFFu;
        for (uint32_t j = lane; j < c; j += 32) {
            uint32_t nbr = ids[i * K + j];
            if ((hdr[nbr] & 0xFFFFu) == 0) continue;
            if (dist[i * K + j] > worst_of(hdr, dist, K, nbr))
                atomicAdd(&rcount[2 * (size_t)nbr + (isnew[i * K + j] ? 0 : 1)], 1u);
        }
    }
}

// Forward samples (first S new / first S old by rank), reverse-candidate scatter,
// and clearing of the new flags.
__global__ void k_sample_fill(const uint32_t* __restrict__ ids, const float* __restrict__ dist,
                              const uint32_t* __restrict__ hdr, uint8_t* __restrict__ isnew, uint32_t n, uint32_t K,
                              uint32_t S, uint32_t cap, uint32_t* __restrict__ newl, uint32_t* __restrict__ newc,
                              uint32_t* __restrict__ oldl, uint32_t* __restrict__ oldc,
                              const uint64_t* __restrict__ roff, uint32_t* __restrict__ rcur,
                              uint32_t* __restrict__ rbuf) {
    size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t i = warp; i < n; i += nw) {
        uint32_t c = hdr[i] & 0xFFFFu;
        uint32_t nn = 0, no = 0;
        for (uint32_t base = 0; base < c; base += 32) {
            uint32_t j = base + lane;
            bool valid = j < c;
            uint32_t nbr = valid ? ids[i * K + j] : 0;
            bool isn = valid && isnew[i * K + j];
            uint32_t bn = __ballot_sync(0xFFFFFFFFu, isn);
            uint32_t bo = __ballot_sync(0xFFFFFFFFu, valid && !isn);
            if (isn) {
                uint32_t r = nn + __popc(bn & lanemask_lt_());
                if (r < S) newl[i * cap + r] = nbr;
                isnew[i * K + j] = 0;
            } else if (valid) {
                uint32_t r = no + __popc(bo & lanemask_lt_());
                if (r < S) oldl[i * cap + r] = nbr;
            }
            nn += __popc(bn);
            no += __popc(bo);
            if (valid && (hdr[nbr] & 0xFFFFu) != 0 && dist[i * K + j] > worst_of(hdr, dist, K, nbr)) {
                size_t seg = 2 * (size_t)nbr + (isn ? 0 : 1);
                rbuf[roff[seg] + atomicAdd(&rcur[seg], 1u)] = (uint32_t)i;
            }
        }
        if (lane == 0) {
            newc[i] = min(nn, S);
            oldc[i] = min(no, S);
        }
    }
}

// Appends the R smallest owners of each reverse segment, ascending, after the
// forward samples (nn_old then stays within 2R = S + R, hrnn.h:1816-1817).
__global__ void k_sample_rev(uint32_t n, uint32_t R, uint32_t cap, const uint64_t* __restrict__ roff,
                             const uint32_t* __restrict__ rbuf, uint32_t* __restrict__ newl,
                             uint32_t* __restrict__ newc, uint32_t* __restrict__ oldl, uint32_t* __restrict__ oldc) {
    size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t i = warp; i < n; i += nw) {
        for (int type = 0; type < 2; ++type) {
            size_t seg = 2 * i + type;
            uint64_t b = roff[seg], e = roff[seg + 1];
            uint32_t len = (uint32_t)(e - b);
            uint32_t* L = type == 0 ? newl : oldl;
            uint32_t* C = type == 0 ? newc : oldc;
            uint32_t base = C[i];
            uint32_t take = min(len, R);
            // R smallest owners, ascending: `take` rounds of a warp minimum above the
            // previous pick (owners are distinct within a segment).
            long long last = -1;
            for (uint32_t r = 0; r < take; ++r) {
                uint32_t mn = kInvalid;
                for (uint32_t x = lane; x < len; x += 32) {
                    uint32_t v = rbuf[b + x];
                    if ((long long)v > last && v < mn) mn = v;
                }
                for (int o = 16; o; o >>= 1) mn = min(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, o));
                if (lane == 0) L[i * cap + base + r] = mn;
                last = mn;
            }
            __syncwarp();
            if (lane == 0) C[i] = base + take;
        }
    }
}

// ---- phase 2: join -----------------------------------------------------------

struct Prop {
    uint32_t target, source;
    float d;
};

// One block per node of the chunk: exact FP32 distances of all sample pairs,
// staged in shared memory (rows padded by one float against bank conflicts).
template <bool FUSED>
__global__ void __launch_bounds__(256) k_join(const float* __restrict__ vec, uint32_t dim, uint32_t node0,
                                              uint32_t node1, uint32_t cap, const uint32_t* __restrict__ newl,
                                              const uint32_t* __restrict__ newc, const uint32_t* __restrict__ oldl,
                                              const uint32_t* __restrict__ oldc, const float* __restrict__ thr,
                                              Prop* __restrict__ prop, unsigned long long* __restrict__ pcount,
                                              unsigned long long pcap, unsigned long long* __restrict__ njoin) {
    extern __shared__ float sm[];
    const uint32_t stride = dim + 1;
    uint32_t* sid = (uint32_t*)(sm + (size_t)2 * cap * stride);
    float* sthr = (float*)(sid + 2 * cap);
    const int lane = threadIdx.x & 31;
    unsigned long long local_pairs = 0;
    for (uint32_t node = node0 + blockIdx.x; node < node1; node += gridDim.x) {
        const uint32_t nn = newc[node], no = oldc[node];
        if (nn == 0) continue;  // no pairs (uniform over the block)
        const uint32_t tot = nn + no;
        __syncthreads();
        for (uint32_t r = threadIdx.x; r < tot; r += blockDim.x) {
            uint32_t id = r < nn ? newl[(size_t)node * cap + r] : oldl[(size_t)node * cap + (r - nn)];
            sid[r] = id;
            sthr[r] = thr[id];
        }
        __syncthreads();
        for (uint32_t idx = threadIdx.x; idx < tot * dim; idx += blockDim.x) {
            uint32_t r = idx / dim, e = idx % dim;
            sm[r * stride + e] = vec[(size_t)sid[r] * dim + e];
        }
        __syncthreads();
        // rows i in [0, nn); partners j in (i, tot): j < nn is new x new, j >= nn new x old.
        // Pair t -> (i, j) through the row offsets off(i) = sum_{i'<i} (tot-1-i')
        // = i (tot-1) - i (i-1) / 2.
        auto rowoff = [tot](uint32_t i) { return i * (tot - 1) - i * (i - 1) / 2; };
        const uint32_t T = rowoff(nn);
        for (uint32_t t0 = 0; t0 < T; t0 += blockDim.x) {
            const uint32_t t = t0 + threadIdx.x;
            bool emit_a = false, emit_b = false;
            uint32_t a = 0, b = 0;
            float d = 0.f;
            if (t < T) {
                uint32_t lo = 0, hi = nn;  // last row with rowoff <= t
                while (hi - lo > 1) {
                    uint32_t mid = (lo + hi) >> 1;
                    if (rowoff(mid) <= t) lo = mid;
                    else hi = mid;
                }
                const uint32_t i = lo, j = i + 1 + (t - rowoff(i));
                a = sid[i];
                b = sid[j];
                if (a != b) {
                    const float* va = sm + (size_t)i * stride;
                    const float* vb = sm + (size_t)j * stride;
                    float acc[16];
#pragma unroll
                    for (int l = 0; l < 16; ++l) acc[l] = 0.f;
                    for (uint32_t e = 0; e < dim; e += 16) {
#pragma unroll
                        for (int l = 0; l < 16; ++l) acc[l] = sq_step(acc[l], va[e + l] - vb[e + l], FUSED);
                    }
                    d = acc[0];
#pragma unroll
                    for (int l = 1; l < 16; ++l) d = __fadd_rn(d, acc[l]);
                    local_pairs++;
                    emit_a = d < sthr[i];
                    emit_b = d < sthr[j];
                }
            }
            // warp-aggregated append
            const uint32_t ba = __ballot_sync(0xFFFFFFFFu, emit_a), bb = __ballot_sync(0xFFFFFFFFu, emit_b);
            const uint32_t tot_w = __popc(ba) + __popc(bb);
            if (tot_w) {
                unsigned long long basep = 0;
                if (lane == 0) basep = atomicAdd(pcount, (unsigned long long)tot_w);
                basep = __shfl_sync(0xFFFFFFFFu, basep, 0);
                unsigned long long p = basep + __popc(ba & lanemask_lt_()) + __popc(bb & lanemask_lt_());
                if (emit_a) {
                    if (p < pcap) prop[p] = Prop{a, b, d};
                    p++;
                }
                if (emit_b && p < pcap) prop[p] = Prop{b, a, d};
            }
        }
    }
    atomicAdd(njoin, local_pairs);
}

// Generic-dim fallback (dims not a multiple of 16, or 8/4-lane orders): one thread
// per pair reading global memory.
__global__ void k_join_generic(const float* __restrict__ vec, uint32_t dim, int lanes, int fused, uint32_t node0,
                               uint32_t node1, uint32_t cap, const uint32_t* __restrict__ newl,
                               const uint32_t* __restrict__ newc, const uint32_t* __restrict__ oldl,
                               const uint32_t* __restrict__ oldc, const float* __restrict__ thr,
                               Prop* __restrict__ prop, unsigned long long* __restrict__ pcount,
                               unsigned long long pcap, unsigned long long* __restrict__ njoin) {
    unsigned long long local_pairs = 0;
    for (uint32_t node = node0 + blockIdx.x; node < node1; node += gridDim.x) {
        const uint32_t nn = newc[node], no = oldc[node], tot = nn + no;
        auto idof = [&](uint32_t r) { return r < nn ? newl[(size_t)node * cap + r] : oldl[(size_t)node * cap + r - nn]; };
        for (uint32_t i = 0; i < nn; ++i) {
            const uint32_t a = idof(i);
            for (uint32_t j = i + 1 + threadIdx.x; j < tot; j += blockDim.x) {
                const uint32_t b = idof(j);
                if (a == b) continue;
                float d = l2_thread(vec + (size_t)a * dim, vec + (size_t)b * dim, dim, lanes, fused);
                local_pairs++;
                bool ea = d < thr[a], eb = d < thr[b];
                uint32_t cnt = (uint32_t)ea + (uint32_t)eb;
                if (cnt) {
                    unsigned long long p = atomicAdd(pcount, (unsigned long long)cnt);
                    if (ea && p < pcap) prop[p++] = Prop{a, b, d};
                    if (eb && p < pcap) prop[p] = Prop{b, a, d};
                }
            }
        }
    }
    atomicAdd(njoin, local_pairs);
}

__global__ void k_thresholds(const uint32_t* __restrict__ hdr, const float* __restrict__ dist, uint32_t n, uint32_t K,
                             float* __restrict__ thr) {
    uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u < n) thr[u] = worst_of(hdr, dist, K, u);
}

__global__ void k_bucket_count(const Prop* __restrict__ prop, unsigned long long np, uint32_t* __restrict__ tcount) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x)
        atomicAdd(&tcount[prop[i].target], 1u);
}

__global__ void k_bucket_fill(const Prop* __restrict__ prop, unsigned long long np, const uint64_t* __restrict__ toff,
                              uint32_t* __restrict__ tcur, uint64_t* __restrict__ bucket) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
        Prop p = prop[i];
        uint64_t pos = toff[p.target] + atomicAdd(&tcur[p.target], 1u);
        bucket[pos] = ((uint64_t)__float_as_uint(p.d) << 32) | p.source;  // d >= 0: bit order = value order
    }
}

// ---- phase 2: merge ----------------------------------------------------------

constexpr int kMergeWarps = 4;
constexpr uint32_t kPiece = 1024;

// Shared memory of one merge warp: keys (u64, first, so 8-byte alignment needs a
// per-warp stride that is a multiple of 8), the list twice (d, id, flag), the id
// table.  Rounded up to 16 bytes.
__host__ __device__ inline size_t merge_warp_bytes(uint32_t K, uint32_t hcap) {
    size_t b = (size_t)K * 18 + (size_t)kPiece * 8 + (size_t)hcap * 4 + 64;
    return (b + 15) & ~(size_t)15;
}

__device__ __forceinline__ uint32_t hmix(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    return x;
}

// One warp per target with proposals.  Shared memory per warp: the list (d, id,
// flag) twice, a piece of sorted proposal keys and an id hash of the list.
__global__ void __launch_bounds__(kMergeWarps * 32) k_merge(uint32_t n, uint32_t K, const uint64_t* __restrict__ toff,
                                                           const uint64_t* __restrict__ bucket,
                                                           uint32_t* __restrict__ hdr, uint32_t* __restrict__ ids,
                                                           float* __restrict__ dist, uint8_t* __restrict__ isnew,
                                                           uint32_t hcap, unsigned long long* __restrict__ nupd) {
    extern __shared__ char smraw[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const size_t per_warp = merge_warp_bytes(K, hcap);  // multiple of 16: the u64 keys stay aligned
    char* base = smraw + w * per_warp;
    uint64_t* keys = (uint64_t*)base;
    float* Ld = (float*)(keys + kPiece);
    uint32_t* Li = (uint32_t*)(Ld + K);
    float* Ld2 = (float*)(Li + K);
    uint32_t* Li2 = (uint32_t*)(Ld2 + K);
    uint32_t* hs = Li2 + K;
    uint8_t* Lf = (uint8_t*)(hs + hcap);
    uint8_t* Lf2 = Lf + K;
    unsigned long long upd = 0;
    for (size_t u = (size_t)blockIdx.x * kMergeWarps + w; u < n; u += (size_t)gridDim.x * kMergeWarps) {
        const uint64_t pb = toff[u], pe = toff[u + 1];
        if (pb == pe) continue;
        uint32_t cnt = hdr[u] & 0xFFFFu;
        for (uint32_t j = lane; j < cnt; j += 32) {
            Ld[j] = dist[u * K + j];
            Li[j] = ids[u * K + j];
            Lf[j] = isnew[u * K + j];
        }
        uint32_t lo_written = cnt;  // first list position that changed
        for (uint64_t p0 = pb; p0 < pe; p0 += kPiece) {
            const uint32_t P = (pe - p0) < kPiece ? (uint32_t)(pe - p0) : kPiece;
            uint32_t PP = 32;
            while (PP < P) PP <<= 1;
            for (uint32_t x = lane; x < PP; x += 32) keys[x] = x < P ? bucket[p0 + x] : ~0ull;
            for (uint32_t x = lane; x < hcap; x += 32) hs[x] = kInvalid;
            __syncwarp();
            for (uint32_t j = lane; j < cnt; j += 32) {  // id hash of the current list
                uint32_t id = Li[j], s = hmix(id) & (hcap - 1);
                while (atomicCAS(&hs[s], kInvalid, id) != kInvalid) s = (s + 1) & (hcap - 1);
            }
            // bitonic sort of the piece by (d, source)
            for (uint32_t k = 2; k <= PP; k <<= 1)
                for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                    __syncwarp();
                    for (uint32_t x = lane; x < PP; x += 32) {
                        uint32_t y = x ^ j;
                        if (y > x) {
                            uint64_t a = keys[x], b = keys[y];
                            if ((a > b) == ((x & k) == 0)) {
                                keys[x] = b;
                                keys[y] = a;
                            }
                        }
                    }
                }
            __syncwarp();
            const float worst = cnt >= K ? Ld[cnt - 1] : FLT_MAX;
            // keep: first of equal sources, not already listed, below the farthest
            // entry when the list is full.  Compact kept keys to the front.
            uint32_t kept = 0;
            uint64_t carry = ~0ull;  // last original key of the previous group of 32
            for (uint32_t x0 = 0; x0 < P; x0 += 32) {
                uint32_t x = x0 + lane;
                bool keep = false;
                uint64_t kx = x < P ? keys[x] : ~0ull;
                uint64_t prev = __shfl_up_sync(0xFFFFFFFFu, kx, 1);
                if (lane == 0) prev = carry;
                carry = __shfl_sync(0xFFFFFFFFu, kx, 31);
                if (x < P) {
                    uint32_t src = (uint32_t)kx;
                    float d = __uint_as_float((uint32_t)(kx >> 32));
                    keep = (x == 0 || prev != kx) && d < worst;
                    if (keep) {
                        uint32_t s = hmix(src) & (hcap - 1);
                        while (hs[s] != kInvalid) {
                            if (hs[s] == src) {
                                keep = false;
                                break;
                            }
                            s = (s + 1) & (hcap - 1);
                        }
                    }
                }
                uint32_t b = __ballot_sync(0xFFFFFFFFu, keep);
                __syncwarp();
                if (keep) keys[kept + __popc(b & lanemask_lt_())] = kx;
                kept += __popc(b);
                __syncwarp();
            }
            if (kept == 0) continue;
            // merge list (cnt) with kept (sorted) -> K; ties: list entries first
            const uint32_t ncnt = min(cnt + kept, K);
            uint32_t lo = 0xFFFFFFFFu;
            for (uint32_t j = lane; j < cnt; j += 32) {
                float d = Ld[j];
                uint32_t l2 = 0, h2 = kept;  // kept entries with distance < d
                while (l2 < h2) {
                    uint32_t mid = (l2 + h2) >> 1;
                    if (__uint_as_float((uint32_t)(keys[mid] >> 32)) < d) l2 = mid + 1;
                    else h2 = mid;
                }
                uint32_t pos = j + l2;
                if (pos < ncnt) {
                    Ld2[pos] = d;
                    Li2[pos] = Li[j];
                    Lf2[pos] = Lf[j];
                }
                if (l2 > 0) lo = min(lo, j);
            }
            for (uint32_t x = lane; x < kept; x += 32) {
                float d = __uint_as_float((uint32_t)(keys[x] >> 32));
                uint32_t l2 = 0, h2 = cnt;  // list entries with distance <= d
                while (l2 < h2) {
                    uint32_t mid = (l2 + h2) >> 1;
                    if (Ld[mid] <= d) l2 = mid + 1;
                    else h2 = mid;
                }
                uint32_t pos = x + l2;
                if (pos < ncnt) {
                    Ld2[pos] = d;
                    Li2[pos] = (uint32_t)keys[x];
                    Lf2[pos] = 1;
                    lo = min(lo, pos);
                    upd++;
                }
            }
            for (int o = 16; o; o >>= 1) lo = min(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, o));
            __syncwarp();
            for (uint32_t j = lane; j < ncnt; j += 32) {
                Ld[j] = Ld2[j];
                Li[j] = Li2[j];
                Lf[j] = Lf2[j];
            }
            cnt = ncnt;
            lo_written = min(lo_written, lo);
            __syncwarp();
        }
        for (uint32_t j = lo_written + lane; j < cnt; j += 32) {
            dist[u * K + j] = Ld[j];
            ids[u * K + j] = Li[j];
            isnew[u * K + j] = Lf[j];
        }
        if (lane == 0) hdr[u] = (hdr[u] & 0xFFFF0000u) | cnt;
        __syncwarp();
    }
    atomicAdd(nupd, upd);
}

int smcount(int dev) {
    int v = 148;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v;
}

}  // namespace

void refine_knng(Index& ix, int iters, int sample) {
    const uint32_t n = (uint32_t)ix.cur, K = (uint32_t)ix.K;
    if (K == 0) fail(HRNN_ERR_STATE, "refineKNNG: index has no KNN graph slot (K_knng = 0)");
    if (K > kMaxK) fail(HRNN_ERR_ARG, "refineKNNG: K_knng above 2048 is not supported");
    if (ix.serve_mode) fail(HRNN_ERR_STATE, "refineKNNG: KNN graph slot removed by compactForServing");
    if (sample <= 0 || iters < 0) fail(HRNN_ERR_ARG, "refineKNNG: sample must be > 0");
    std::printf("    refineKNNG (NNDescent, device): n=%u K=%u iters=%d S=%d\n", n, K, iters, sample);
    const uint32_t S = (uint32_t)sample, R = S, cap = S + R;
    cudaStream_t s = ix.stream;
    if (n == 0) {
        ix.knng_built = true;
        return;
    }
    const int nsm = smcount(ix.device);
    // Device state of the refinement.
    DevMem isnew, newl, newc, oldl, oldc, rcount, roff, rcur, rbuf, thr, prop, tcount, toff, tcur, bucket, tmp, ctr;
    isnew.alloc((size_t)n * K + 16);
    // INIT (hrnn.h:1744-1748): every existing entry is new.
    if (n) {
        size_t tot = (size_t)n * K;
        k_init_flags<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(ix.knn_hdr.as<uint32_t>(), n, K,
                                                                   isnew.as<uint8_t>());
        CUDA_LAUNCH_CHECK();
    }
    newl.alloc((size_t)n * cap * 4);
    oldl.alloc((size_t)n * cap * 4);
    newc.alloc((size_t)n * 4);
    oldc.alloc((size_t)n * 4);
    rcount.alloc(((size_t)2 * n + 1) * 4);
    roff.alloc(((size_t)2 * n + 1) * 8);
    rcur.alloc(((size_t)2 * n + 1) * 4);
    thr.alloc((size_t)n * 4);
    tcount.alloc(((size_t)n + 1) * 4);
    toff.alloc(((size_t)n + 1) * 8);
    tcur.alloc(((size_t)n + 1) * 4);
    ctr.alloc(64);
    const unsigned long long pcap = std::max<unsigned long long>(1 << 20, std::min<unsigned long long>(
                                                                              400ull << 20, (unsigned long long)n * 512));
    prop.alloc(pcap * sizeof(Prop));
    bucket.alloc(pcap * 8);
    uint32_t* hdr = ix.knn_hdr.as<uint32_t>();
    uint32_t* ids = ix.knn_ids.as<uint32_t>();
    float* dist = ix.knn_dist.as<float>();
    unsigned long long* d_pcount = ctr.as<unsigned long long>();
    unsigned long long* d_njoin = d_pcount + 1;
    unsigned long long* d_nupd = d_pcount + 2;
    const bool fast = ix.order.lanes == 16 && ix.dim % 16 == 0;
    const size_t join_smem = (size_t)2 * cap * (ix.dim + 1) * 4 + (size_t)2 * cap * 8;
    if (fast) {
        auto kj = (ix.order.fused & 1) ? k_join<true> : k_join<false>;
        if (join_smem > 227 * 1024) fail(HRNN_ERR_ARG, "refineKNNG: sample size too large for dim");
        CUDA_CHECK(cudaFuncSetAttribute(kj, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)join_smem));
    }
    uint32_t hcap = 64;
    while (hcap < 2 * K) hcap <<= 1;
    const size_t merge_smem = (size_t)kMergeWarps * merge_warp_bytes(K, hcap);
    if (merge_smem > 227 * 1024) fail(HRNN_ERR_ARG, "refineKNNG: K_knng too large for the merge kernel");
    CUDA_CHECK(cudaFuncSetAttribute(k_merge, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)merge_smem));
    const int g1 = nsm * 16;
    ix.refine_stats = hrnn_refine_stats{};
    // Events bracketing sampling, and each chunk's join and bucket+merge.
    cudaEvent_t ev[7];
    for (auto& e : ev) CUDA_CHECK(cudaEventCreate(&e));
    auto elapsed = [](cudaEvent_t a, cudaEvent_t b) {
        float t = 0.f;
        cudaEventElapsedTime(&t, a, b);
        return (double)t;
    };
    for (int it = 0; it < iters; ++it) {
        cudaEvent_t e0 = ev[0], e1 = ev[1];
        double t_join = 0, t_bucket = 0, t_merge = 0, t_sample = 0;
        CUDA_CHECK(cudaEventRecord(e0, s));
        CUDA_CHECK(cudaMemsetAsync(ctr.p, 0, 64, s));
        // ---- phase 1 ----
        CUDA_CHECK(cudaMemsetAsync(rcount.p, 0, rcount.bytes, s));
        CUDA_CHECK(cudaMemsetAsync(rcur.p, 0, rcur.bytes, s));
        k_sample_count<<<g1, 256, 0, s>>>(ids, dist, hdr, isnew.as<uint8_t>(), n, K, rcount.as<uint32_t>());
        CUDA_LAUNCH_CHECK();
        exclusive_scan_u32_to_u64(rcount.as<uint32_t>(), roff.as<uint64_t>(), (size_t)2 * n + 1, s, tmp);
        uint64_t rtot = 0;
        CUDA_CHECK(cudaMemcpyAsync(&rtot, roff.as<uint64_t>() + (size_t)2 * n, 8, cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaStreamSynchronize(s));
        rbuf.ensure(std::max<uint64_t>(rtot, 1) * 4);
        k_sample_fill<<<g1, 256, 0, s>>>(ids, dist, hdr, isnew.as<uint8_t>(), n, K, S, cap, newl.as<uint32_t>(),
                                          newc.as<uint32_t>(), oldl.as<uint32_t>(), oldc.as<uint32_t>(),
                                          roff.as<uint64_t>(), rcur.as<uint32_t>(), rbuf.as<uint32_t>());
        CUDA_LAUNCH_CHECK();
        k_sample_rev<<<g1, 256, 0, s>>>(n, R, cap, roff.as<uint64_t>(), rbuf.as<uint32_t>(), newl.as<uint32_t>(),
                                         newc.as<uint32_t>(), oldl.as<uint32_t>(), oldc.as<uint32_t>());
        CUDA_LAUNCH_CHECK();
        CUDA_CHECK(cudaEventRecord(ev[2], s));
        // |new| + |old| summed over nodes (gather bytes of the join)
        unsigned long long sample_entries = 0;
        {
            std::vector<uint32_t> a(n), b(n);
            CUDA_CHECK(cudaMemcpyAsync(a.data(), newc.p, (size_t)n * 4, cudaMemcpyDeviceToHost, s));
            CUDA_CHECK(cudaMemcpyAsync(b.data(), oldc.p, (size_t)n * 4, cudaMemcpyDeviceToHost, s));
            CUDA_CHECK(cudaStreamSynchronize(s));
            for (uint32_t i = 0; i < n; ++i) sample_entries += (unsigned long long)a[i] + b[i];
            t_sample = elapsed(e0, ev[2]);
        }
        unsigned long long proposals = 0;
        // ---- phase 2, chunk by chunk ----
        uint32_t chunk = std::max<uint32_t>(1, std::min<uint32_t>(n, 4096));
        for (uint32_t node0 = 0; node0 < n;) {
            uint32_t node1 = std::min<uint32_t>(n, node0 + chunk);
            k_thresholds<<<(n + 255) / 256, 256, 0, s>>>(hdr, dist, n, K, thr.as<float>());
            CUDA_LAUNCH_CHECK();
            CUDA_CHECK(cudaMemsetAsync(d_pcount, 0, 8, s));
            CUDA_CHECK(cudaEventRecord(ev[3], s));
            unsigned grid = std::min<unsigned>(node1 - node0, (unsigned)nsm * 8);
            if (fast) {
                auto kj = (ix.order.fused & 1) ? k_join<true> : k_join<false>;
                kj<<<grid, 256, join_smem, s>>>(ix.vec.as<float>(), (uint32_t)ix.dim, node0, node1, cap,
                                                newl.as<uint32_t>(), newc.as<uint32_t>(), oldl.as<uint32_t>(),
                                                oldc.as<uint32_t>(), thr.as<float>(), prop.as<Prop>(), d_pcount, pcap,
                                                d_njoin);
            } else {
                k_join_generic<<<grid, 128, 0, s>>>(ix.vec.as<float>(), (uint32_t)ix.dim, ix.order.lanes,
                                                    ix.order.fused, node0, node1, cap, newl.as<uint32_t>(),
                                                    newc.as<uint32_t>(), oldl.as<uint32_t>(), oldc.as<uint32_t>(),
                                                    thr.as<float>(), prop.as<Prop>(), d_pcount, pcap, d_njoin);
            }
            CUDA_LAUNCH_CHECK();
            CUDA_CHECK(cudaEventRecord(ev[4], s));
            unsigned long long np = 0;
            CUDA_CHECK(cudaMemcpyAsync(&np, d_pcount, 8, cudaMemcpyDeviceToHost, s));
            CUDA_CHECK(cudaStreamSynchronize(s));
            t_join += elapsed(ev[3], ev[4]);
            if (np > pcap) {
                if (chunk == 1) fail(HRNN_ERR_NOMEM, "refineKNNG: proposal buffer too small for one node");
                chunk = std::max<uint32_t>(1, chunk / 4);  // redo this chunk smaller (the join is pure)
                unsigned long long z = 0;
                CUDA_CHECK(cudaMemcpyAsync(d_njoin, &z, 8, cudaMemcpyHostToDevice, s));
                continue;
            }
            if (np) {
                CUDA_CHECK(cudaMemsetAsync(tcount.p, 0, tcount.bytes, s));
                CUDA_CHECK(cudaMemsetAsync(tcur.p, 0, tcur.bytes, s));
                unsigned gb = (unsigned)std::min<unsigned long long>((np + 255) / 256, (unsigned long long)nsm * 32);
                k_bucket_count<<<gb, 256, 0, s>>>(prop.as<Prop>(), np, tcount.as<uint32_t>());
                CUDA_LAUNCH_CHECK();
                exclusive_scan_u32_to_u64(tcount.as<uint32_t>(), toff.as<uint64_t>(), (size_t)n + 1, s, tmp);
                k_bucket_fill<<<gb, 256, 0, s>>>(prop.as<Prop>(), np, toff.as<uint64_t>(), tcur.as<uint32_t>(),
                                                 bucket.as<uint64_t>());
                CUDA_LAUNCH_CHECK();
                CUDA_CHECK(cudaEventRecord(ev[6], s));
                k_merge<<<nsm * 4, kMergeWarps * 32, merge_smem, s>>>(n, K, toff.as<uint64_t>(),
                                                                      bucket.as<uint64_t>(), hdr, ids, dist,
                                                                      isnew.as<uint8_t>(), hcap, d_nupd);
                CUDA_LAUNCH_CHECK();
                CUDA_CHECK(cudaEventRecord(ev[5], s));
                CUDA_CHECK(cudaEventSynchronize(ev[5]));
                t_bucket += elapsed(ev[4], ev[6]);
                t_merge += elapsed(ev[6], ev[5]);
            }
            proposals += np;
            node0 = node1;
            // Grow the chunk while proposals stay well inside the buffer.
            if (np < pcap / 8 && chunk < n) chunk = std::min<uint32_t>(n, chunk * 2);
        }
        unsigned long long hc[3] = {0, 0, 0};
        CUDA_CHECK(cudaEventRecord(e1, s));
        CUDA_CHECK(cudaMemcpyAsync(hc, ctr.p, 24, cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaStreamSynchronize(s));
        const double ms = elapsed(e0, e1);
        std::printf("      iter %d: %llu updates, %llu dists  (%.1f ms: sample %.1f, join %.1f, bucket %.1f, "
                    "merge %.1f)\n", it, hc[2], hc[1], ms, t_sample, t_join, t_bucket, t_merge);
        std::fflush(stdout);
        if (it < HRNN_MAX_ITERS) {
            auto& rs = ix.refine_stats;
            rs.iters = it + 1;
            rs.join_dists[it] = hc[1];
            rs.updates[it] = hc[2];
            rs.proposals[it] = proposals;
            rs.sample_entries[it] = sample_entries;
            rs.ms[it] = ms;
            rs.sample_ms[it] = t_sample;
            rs.join_ms[it] = t_join;
            rs.bucket_ms[it] = t_bucket;
            rs.merge_ms[it] = t_merge;
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    ix.knng_built = true;                                 // hrnn.h:1861
}

}  // namespace hrnn
