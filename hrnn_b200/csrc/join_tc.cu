// Local join of NNDescent (refineKNNG phase 2, hrnn.h:1823-1853) screened on the
// tensor cores.
//
// The join of a node compares every new x new (i < j) and new x old pair of its
// sample lists; a pair becomes a proposal for target a when its exact FP32
// distance is below a's current farthest entry (thr[a], FLT_MAX while the list is
// not full).  Most pairs of a converging graph are proposals for neither end.
// This kernel decides that for most pairs from a BF16 Gram matrix and computes the
// exact FP32 distance (the reference's summation order) only for the rest, so the
// proposals -- and hence the lists -- are exactly those of the exact join.
//
// One CTA of 512 threads per node at a time (persistent over the chunk):
//   1. the node's rows (new first, then old; at most 256) are gathered as FP32 into
//      shared memory (stride dim + 4 floats);
//   2. from them, the BF16 tile in the canonical K-major no-swizzle layout (8-row x
//      16-byte core matrices, K-adjacent core matrices 128 bytes apart, 8-row groups
//      16 * dim bytes apart), the FP32 squared norm n(r) of each BF16 row and the
//      rounding error e(r) >= ||x_r - bf16(x_r)||;
//   3. one thread issues dim / 16 tcgen05.mma (M = 128 new rows, N = the node's
//      rows rounded up to 16, K = 16; A and B both read from the same tile) into
//      an FP32 accumulator in TMEM and commits them to an mbarrier (bounded wait);
//   4. warp w reads TMEM lanes 32 (w mod 4) .. +31 (rows i), columns of its
//      quarter, and for each pair forms the lower bound
//          Lb = (max(0, sqrt(max(0, D - E)) - e(i) - e(j)))^2 (1 - rho),
//          D = n(i) + n(j) - 2 G(i, j),  E = cE (sqrt n(i) + sqrt n(j))^2,
//      where E bounds the FP32 rounding of the norms, of the tensor-core sums and
//      of D (cE = (2 dim + 64) 2^-20, 16x the FP32 accumulation bound of dim
//      products), e(i) + e(j) the BF16 rounding of the rows (triangle inequality),
//      and rho the gap between the exact squared distance and the reference's FP32
//      sum plus this bound's own roundings.  A pair with Lb >= max(thr[a], thr[b])
//      cannot be a proposal and is dropped; the others are listed;
//   5. the listed pairs get the exact FP32 distance from the shared-memory rows
//      (16 accumulators, element e into e mod 16, summed left to right) and emit
//      their proposals.  A node whose list overflows runs the dense exact pass
//      over all its pairs instead.
// Audit mode runs steps 1-4, records the screen's decisions in a bitmap, runs the
// dense exact pass and counts proposals the screen would have dropped.
#include <cuda_bf16.h>

#include <algorithm>
#include <cfloat>
#include <cstdint>

#include "common.cuh"
#include "join.cuh"

namespace hrnn {

namespace {

constexpr int kJT = 512;              // threads per CTA (16 warps)
constexpr uint32_t kMaxRows = 256;    // N of the MMA: all rows of a node
constexpr uint32_t kMaxNew = 128;     // M of the MMA: the node's new rows
constexpr uint32_t kSurvCap = 4096;   // listed pairs per node before the dense pass
constexpr uint32_t kWaitLimit = 1u << 26;

struct JtLayout {
    uint32_t SP;  // FP32 row stride in floats
    size_t tile, sid, sthr, sn2, sn, serr, surv, ctl, mbar, total;
};

__host__ __device__ inline JtLayout jt_layout(uint32_t dim, uint32_t cap) {
    JtLayout L;
    L.SP = dim + 4;
    size_t o = (size_t)2 * cap * L.SP * 4;  // FP32 rows at offset 0
    o = (o + 1023) & ~(size_t)1023;
    L.tile = o;
    o += (size_t)kMaxRows * dim * 2;
    L.sid = o;
    o += kMaxRows * 4;
    L.sthr = o;
    o += kMaxRows * 4;
    L.sn2 = o;
    o += kMaxRows * 4;
    L.sn = o;
    o += kMaxRows * 4;
    L.serr = o;
    o += kMaxRows * 4;
    L.surv = o;  // listed pairs (i << 16 | j); audit: the 128 x 256-bit decision map
    o += (size_t)kSurvCap * 4;
    L.ctl = o;   // 0 listed count, 1 overflow, 2 TMEM base
    o += 32;
    L.mbar = o;
    o += 16;
    L.total = o;
    return L;
}

// Byte offset of element (r, k) in the K-major core-matrix layout (sbo = 16 dim).
__device__ __forceinline__ uint32_t cm_off(uint32_t r, uint32_t k, uint32_t sbo) {
    return (r >> 3) * sbo + (k >> 3) * 128u + (r & 7) * 16u + (k & 7) * 2u;
}

// Shared-memory matrix descriptor, K-major, no swizzle: start address, leading
// byte offset 128 (K-adjacent core matrices), stride byte offset sbo, version 1.
__device__ __forceinline__ uint64_t jt_desc(uint32_t saddr, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           (1ull << 46);
}

// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both K-major,
// M = 128, N = n (a multiple of 16, at most 256).
__device__ __forceinline__ uint32_t jt_idesc(uint32_t n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((kMaxNew >> 4) << 24);
}

// Exact FP32 distance of two shared-memory rows in the reference's order.
template <bool FUSED>
__device__ __forceinline__ float exact_pair(const float* ra, const float* rb, uint32_t d4) {
    float acc[16];
#pragma unroll
    for (int l = 0; l < 16; ++l) acc[l] = 0.f;
    const float4* a4 = reinterpret_cast<const float4*>(ra);
    const float4* b4 = reinterpret_cast<const float4*>(rb);
    for (uint32_t e4 = 0; e4 < d4; e4 += 4) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const float4 a = a4[e4 + c], b = b4[e4 + c];
            acc[4 * c + 0] = sq_step(acc[4 * c + 0], a.x - b.x, FUSED);
            acc[4 * c + 1] = sq_step(acc[4 * c + 1], a.y - b.y, FUSED);
            acc[4 * c + 2] = sq_step(acc[4 * c + 2], a.z - b.z, FUSED);
            acc[4 * c + 3] = sq_step(acc[4 * c + 3], a.w - b.w, FUSED);
        }
    }
    float dv = acc[0];
#pragma unroll
    for (int l = 1; l < 16; ++l) dv = __fadd_rn(dv, acc[l]);
    return dv;
}

// Appends the proposals of one pair per lane (emit bit 0: i -> j's source is j,
// target i; bit 1: target j) with one atomic per warp.  All lanes call it.
__device__ __forceinline__ void emit_warp(uint32_t emit, uint32_t ai, uint32_t bj, float dv, Prop* prop,
                                          unsigned long long* pcount, unsigned long long pcap) {
    const int lane = threadIdx.x & 31;
    const uint32_t ne = __popc(emit);
    uint32_t incl = ne;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
    }
    const uint32_t wt = __shfl_sync(0xFFFFFFFFu, incl, 31);
    if (wt == 0) return;
    unsigned long long base = 0;
    if (lane == 31) base = atomicAdd(pcount, (unsigned long long)wt);
    base = __shfl_sync(0xFFFFFFFFu, base, 31);
    unsigned long long p = base + (incl - ne);
    if (emit & 1u) {
        if (p < pcap) prop[p] = Prop{ai, bj, dv};
        p++;
    }
    if (emit & 2u) {
        if (p < pcap) prop[p] = Prop{bj, ai, dv};
    }
}

template <bool FUSED, bool AUDIT>
__global__ void __launch_bounds__(kJT, 1) k_join_tc(const float* __restrict__ vec, uint32_t dim, uint32_t node0,
                                                   uint32_t node1, uint32_t cap, const uint32_t* __restrict__ newl,
                                                   const uint32_t* __restrict__ newc,
                                                   const uint32_t* __restrict__ oldl,
                                                   const uint32_t* __restrict__ oldc, const float* __restrict__ thr,
                                                   Prop* __restrict__ prop, unsigned long long* __restrict__ pcount,
                                                   unsigned long long pcap, unsigned long long* __restrict__ njoin,
                                                   JoinTcCounters* __restrict__ jc) {
    extern __shared__ __align__(1024) char sm[];
    const JtLayout L = jt_layout(dim, cap);
    float* rows = reinterpret_cast<float*>(sm);
    char* tile = sm + L.tile;
    uint32_t* sid = reinterpret_cast<uint32_t*>(sm + L.sid);
    float* sthr = reinterpret_cast<float*>(sm + L.sthr);
    float* sn2 = reinterpret_cast<float*>(sm + L.sn2);
    float* sn = reinterpret_cast<float*>(sm + L.sn);
    float* serr = reinterpret_cast<float*>(sm + L.serr);
    uint32_t* surv = reinterpret_cast<uint32_t*>(sm + L.surv);
    uint32_t* ctl = reinterpret_cast<uint32_t*>(sm + L.ctl);
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + L.mbar);
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const uint32_t SP = L.SP, d4 = dim >> 2, nch = dim >> 3, sbo = dim * 16;
    const float cE = (2.f * (float)dim + 64.f) * 0x1p-20f;
    const float rho = (4.f * (float)dim + 64.f) * 0x1p-24f + 0x1p-20f;

    const uint32_t mbar_a = (uint32_t)__cvta_generic_to_shared(mbar);
    if (w == 0) {
        const uint32_t slot = (uint32_t)__cvta_generic_to_shared(ctl + 2);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(kMaxRows));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar_a));
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = ctl[2];
    uint32_t phase = 0;
    unsigned long long pairs = 0, listed = 0, dense_nodes = 0, misses = 0;

    for (uint32_t node = node0 + blockIdx.x; node < node1; node += gridDim.x) {
        const uint32_t nn = newc[node], no = oldc[node];
        if (nn == 0) continue;  // no pairs (uniform over the block)
        const uint32_t tot = nn + no;
        const uint32_t N = (tot + 15) & ~15u;
        __syncthreads();  // the previous node's readers are done with shared memory
        for (uint32_t r = tid; r < tot; r += kJT) {
            const uint32_t id = r < nn ? newl[(size_t)node * cap + r] : oldl[(size_t)node * cap + (r - nn)];
            sid[r] = id;
            sthr[r] = thr[id];
        }
        if (AUDIT)
            for (uint32_t x = tid; x < kMaxNew * kMaxRows / 32; x += kJT) surv[x] = 0;
        if (tid == 0) {
            ctl[0] = 0;
            ctl[1] = 0;
        }
        __syncthreads();
        // 1. FP32 rows, a warp per row
        for (uint32_t r = w; r < tot; r += kJT / 32) {
            const float4* src = reinterpret_cast<const float4*>(vec + (size_t)sid[r] * dim);
            float4* dst = reinterpret_cast<float4*>(rows + (size_t)r * SP);
            for (uint32_t c = lane; c < d4; c += 32) dst[c] = __ldg(src + c);
        }
        __syncthreads();
        // 2. BF16 tile, norms, rounding errors: 16 threads per row (rows r, r+1 per
        // warp; N is even, so both halves of a warp agree on r < N)
        for (uint32_t r = (uint32_t)tid >> 4; r < N; r += kJT / 16) {
            const uint32_t c = (uint32_t)tid & 15u;
            float n2 = 0.f, e2 = 0.f;
            if (c < nch) {
                uint4 wv = make_uint4(0u, 0u, 0u, 0u);
                if (r < tot) {
                    const float4 a = *reinterpret_cast<const float4*>(rows + (size_t)r * SP + 8 * c);
                    const float4 b = *reinterpret_cast<const float4*>(rows + (size_t)r * SP + 8 * c + 4);
                    const float x[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
                    uint32_t pk[4];
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const __nv_bfloat162 h = __floats2bfloat162_rn(x[2 * k], x[2 * k + 1]);
                        pk[k] = *reinterpret_cast<const uint32_t*>(&h);
                        const float b0 = __low2float(h), b1 = __high2float(h);
                        n2 = __fmaf_rn(b0, b0, n2);
                        n2 = __fmaf_rn(b1, b1, n2);
                        const float t0 = x[2 * k] - b0, t1 = x[2 * k + 1] - b1;  // exact (Sterbenz)
                        e2 = __fmaf_rn(t0, t0, e2);
                        e2 = __fmaf_rn(t1, t1, e2);
                    }
                    wv = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                }
                *reinterpret_cast<uint4*>(tile + cm_off(r, 8 * c, sbo)) = wv;
            }
#pragma unroll
            for (int o = 8; o; o >>= 1) {
                n2 += __shfl_xor_sync(0xFFFFFFFFu, n2, o);
                e2 += __shfl_xor_sync(0xFFFFFFFFu, e2, o);
            }
            if (c == 0 && r < tot) {
                sn2[r] = n2;
                sn[r] = sqrtf(n2);
                // e2 carries at most dim roundings of 2^-24 relative: (1 + 2^-14) covers dim <= 1024
                serr[r] = sqrtf(e2 * (1.f + 0x1p-14f)) * (1.f + 0x1p-22f);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic stores -> tensor-core reads
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // 3. the Gram matrix of the new rows against all rows
        if (tid == 0) {
            const uint32_t t0 = (uint32_t)__cvta_generic_to_shared(tile);
            const uint32_t idesc = jt_idesc(N);
#pragma unroll 1
            for (uint32_t s = 0; s < dim / 16; ++s) {
                const uint64_t da = jt_desc(t0 + s * 256u, sbo);
                const uint32_t accum = s > 0 ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(da), "r"(idesc), "r"(accum));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar_a)
                         : "memory");
        }
        uint32_t done = 0;
        for (uint32_t it = 0; it < kWaitLimit && !done; ++it) {
            asm volatile(
                "{\n\t.reg .pred q;\n\tmbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, q;\n\t}\n"
                : "=r"(done)
                : "r"(mbar_a), "r"(phase)
                : "memory");
        }
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (__syncthreads_or(!done)) {
            if (tid == 0) atomicExch(&jc->err, 1);
            break;
        }
        // 4. screen: warp w reads rows 32 (w mod 4) + lane, its quarter of the columns
        {
            const uint32_t q = (uint32_t)w & 3u, cg = (uint32_t)w >> 2;
            const uint32_t i = 32 * q + lane;
            const bool row_ok = i < nn;
            const float ni2 = row_ok ? sn2[i] : 0.f, ni = row_ok ? sn[i] : 0.f, ei = row_ok ? serr[i] : 0.f;
            const float ti = row_ok ? sthr[i] : 0.f;
            const uint32_t ai = row_ok ? sid[i] : 0u;
#pragma unroll 1
            for (uint32_t t = 0; t < 4; ++t) {
                const uint32_t c0 = 64 * cg + 16 * t;
                // uniform over the warp: columns staged, some row of the quarter live,
                // and some column above some row
                if (c0 >= N || 32 * q >= nn || c0 + 15 <= 32 * q) continue;
                uint32_t v[16];
                const uint32_t taddr = tmem + ((32u * q) << 16) + c0;
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                    "[%16];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                      "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                      "=r"(v[14]), "=r"(v[15])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                uint32_t smask = 0;
#pragma unroll
                for (int jj = 0; jj < 16; ++jj) {
                    const uint32_t j = c0 + (uint32_t)jj;
                    if (row_ok && j > i && j < tot && sid[j] != ai) {
                        pairs++;
                        const float G = __uint_as_float(v[jj]);
                        const float D = ni2 + sn2[j] - 2.f * G;
                        const float sum = ni + sn[j];
                        const float E = cE * sum * sum;
                        const float s = sqrtf(fmaxf(D - E, 0.f)) * (1.f - 0x1p-22f);
                        const float tt = fmaxf(s - (ei + serr[j]) * (1.f + 0x1p-22f), 0.f);
                        const float Lb = tt * tt * (1.f - rho);
                        if (Lb < fmaxf(ti, sthr[j])) smask |= 1u << jj;
                    }
                }
                const uint32_t cnt = __popc(smask);
                listed += cnt;
                if (AUDIT) {
                    for (uint32_t m = smask; m; m &= m - 1) {
                        const uint32_t j = c0 + (uint32_t)(__ffs(m) - 1);
                        atomicOr(&surv[i * (kMaxRows / 32) + (j >> 5)], 1u << (j & 31));
                    }
                } else {
                    uint32_t incl = cnt;
                    for (int o = 1; o < 32; o <<= 1) {
                        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                        if (lane >= o) incl += y;
                    }
                    const uint32_t wt = __shfl_sync(0xFFFFFFFFu, incl, 31);
                    uint32_t base = 0;
                    if (lane == 31 && wt) base = atomicAdd(&ctl[0], wt);
                    base = __shfl_sync(0xFFFFFFFFu, base, 31);
                    uint32_t p = base + incl - cnt;
                    for (uint32_t m = smask; m; m &= m - 1, ++p) {
                        const uint32_t j = c0 + (uint32_t)(__ffs(m) - 1);
                        if (p < kSurvCap) surv[p] = (i << 16) | j;
                        else ctl[1] = 1u;
                    }
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        // 5. exact FP32 distances and proposals
        const bool dense = AUDIT || ctl[1] != 0u;
        if (!dense) {
            const uint32_t ns = ctl[0];
            for (uint32_t b0 = (uint32_t)w * 32; b0 < ns; b0 += kJT) {
                const uint32_t k = b0 + lane;
                uint32_t emit = 0, ai = 0, bj = 0;
                float dv = 0.f;
                if (k < ns) {
                    const uint32_t pr = surv[k], i = pr >> 16, j = pr & 0xFFFFu;
                    dv = exact_pair<FUSED>(rows + (size_t)i * SP, rows + (size_t)j * SP, d4);
                    ai = sid[i];
                    bj = sid[j];
                    emit = (dv < sthr[i] ? 1u : 0u) | (dv < sthr[j] ? 2u : 0u);
                }
                emit_warp(emit, ai, bj, dv, prop, pcount, pcap);
            }
        } else {
            if (!AUDIT && tid == 0) dense_nodes++;
            // every pair: a warp per (row i, 32 columns j) tile
            const uint32_t tj_n = (tot + 31) >> 5;
            for (uint32_t t = (uint32_t)w; t < nn * tj_n; t += kJT / 32) {
                const uint32_t i = t / tj_n, jb = (t % tj_n) << 5;
                if (jb + 31 <= i) continue;  // uniform over the warp
                const uint32_t j = jb + lane;
                uint32_t emit = 0, bj = 0;
                float dv = 0.f;
                const uint32_t ai = sid[i];
                if (j > i && j < tot && sid[j] != ai) {
                    bj = sid[j];
                    dv = exact_pair<FUSED>(rows + (size_t)i * SP, rows + (size_t)j * SP, d4);
                    emit = (dv < sthr[i] ? 1u : 0u) | (dv < sthr[j] ? 2u : 0u);
                    if (AUDIT && emit && !((surv[i * (kMaxRows / 32) + (j >> 5)] >> (j & 31)) & 1u)) misses++;
                }
                emit_warp(emit, ai, bj, dv, prop, pcount, pcap);
            }
        }
    }
    // counters
    for (int o = 16; o; o >>= 1) {
        pairs += __shfl_xor_sync(0xFFFFFFFFu, pairs, o);
        listed += __shfl_xor_sync(0xFFFFFFFFu, listed, o);
        misses += __shfl_xor_sync(0xFFFFFFFFu, misses, o);
    }
    if (lane == 0) {
        if (pairs) atomicAdd(njoin, pairs);
        if (listed) atomicAdd(&jc->survivors, listed);
        if (misses) atomicAdd(&jc->misses, misses);
    }
    if (tid == 0 && dense_nodes) atomicAdd(&jc->dense_nodes, dense_nodes);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (w == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kMaxRows));
}

}  // namespace

bool join_tc_supported(uint32_t dim, uint32_t cap) {
    if (dim % 16 != 0 || dim < 16 || dim > 128 || cap == 0 || cap > kMaxNew) return false;
    return jt_layout(dim, cap).total <= 227 * 1024;
}

void join_tc(const float* vec, uint32_t dim, uint32_t node0, uint32_t node1, uint32_t cap, const uint32_t* newl,
             const uint32_t* newc, const uint32_t* oldl, const uint32_t* oldc, const float* thr, Prop* prop,
             unsigned long long* pcount, unsigned long long pcap, unsigned long long* njoin, JoinTcCounters* jc,
             bool fused, int mode, int nsm, cudaStream_t s) {
    if (node1 <= node0) return;
    const JtLayout L = jt_layout(dim, cap);
    // At least 116 KB of shared memory: at most two CTAs per SM, whose 256 TMEM
    // columns each fit the SM's 512, so no allocation waits on another CTA.
    const size_t smem = std::max<size_t>(L.total, 116 * 1024);
    const bool audit = mode == kJoinAudit;
    auto k = fused ? (audit ? k_join_tc<true, true> : k_join_tc<true, false>)
                   : (audit ? k_join_tc<false, true> : k_join_tc<false, false>);
    CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 1;
    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kJT, smem));
    per_sm = std::min(std::max(per_sm, 1), 2);
    const unsigned grid = (unsigned)std::min<size_t>(node1 - node0, (size_t)nsm * per_sm);
    k<<<grid, kJT, smem, s>>>(vec, dim, node0, node1, cap, newl, newc, oldl, oldc, thr, prop, pcount, pcap, njoin,
                              jc);
    CUDA_LAUNCH_CHECK();
}

}  // namespace hrnn
