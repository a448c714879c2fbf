// Warp-level graph search shared by the query path (search.cu) and the batched
// HNSW construction (hnsw_build.cu): greedy descent over the upper layers and
// the best-first beam search of one layer, with the exact FP32 distance order.
//
// Beam formulation of searchBaseLayerST (hrnn.h:484-616): the result max-heap of
// size ef and the candidate min-heap are one ascending list in shared memory
// whose entries carry an "expanded" flag.  The next node to expand is the first
// unexpanded entry; neighbour j of an expansion is accepted iff fewer than ef
// elements of (beam before the expansion + earlier fresh neighbours) are <= d_j,
// which is the reference's sequential test (size < ef || bound > d_j) evaluated
// after the earlier neighbours (neighbours it rejected never change the count).
// The visited array is a lossy direct-mapped cache plus an exact membership test
// against the beam; a point evicted from the cache and met again is either in
// the beam (caught) or was rejected/popped before, in which case the acceptance
// test rejects it again.  Equal distances of different points are the only case
// in which the order can differ from the reference's heaps.
#pragma once

#include <cfloat>

#include "common.cuh"

namespace hrnn {

struct DevView {
    const float* vec;
    const uint32_t* adj0;
    const uint32_t* upper;
    const uint64_t* upper_off;
    const uint32_t* knn_hdr;
    const float* knn_dist;
    const float* kdist_serve;
    const uint64_t* csr_off;
    const void* csr_ent;
    const uint64_t* labels;
    const uint16_t* vec_bf16;  // mixed precision: BF16 rows (or null)
    const float* vec_err;      // ||x - bf16(x)||_2, rounded up
    const uint32_t* knn_ids;   // KNN slot ids (FP64 radius re-decision)
    const int8_t* vec_i8;      // INT8 beam: rows round(x / s) (or null)
    const float4* i8_meta;     // (s, ||x - s c||, sum c^2, 0) per row
    uint32_t n, dim, nb, W0, WU, K, mks, rank_bits;
    int maxlevel;
    uint32_t enterpoint;
    int wide, lanes, fused;
    int i8_screen;             // verification screens with the INT8 rows first
};

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

// Links of node c at `level`: word 0 = count (low 16 bits), then the ids.
__device__ __forceinline__ const uint32_t* links_of(const DevView& v, uint32_t c, int level) {
    if (level == 0) return v.adj0 + (size_t)c * v.W0;
    return v.upper + v.upper_off[c] + (size_t)(level - 1) * v.WU;
}

// Distance of q (shared memory) to one stored vector, by the whole warp.
template <bool FUSED>
__device__ __forceinline__ float warp_l2_one(const DevView& v, const float* q, uint32_t id) {
    int l = threadIdx.x & 15;
    if (v.lanes == 16 && v.dim % 16 == 0) return l2_half16<FUSED>(q, v.vec + (size_t)id * v.dim, v.nb, l);
    return l2_thread(q, v.vec + (size_t)id * v.dim, v.dim, v.lanes, v.fused);
}

// One thread, one row, 16-lane order (the AVX-512 path of space_l2.h:25-54):
// accumulator l takes elements l, l+16, ...; the row is read with 16-byte loads,
// two 64-byte blocks at a time, so a warp keeps up to 32 rows in flight.  q is
// in shared memory (16-byte aligned); every thread reads the same q words.
template <bool FUSED>
__device__ __forceinline__ float l2_row16(const float* __restrict__ q, const float* __restrict__ x, uint32_t nb) {
    float acc[16];
#pragma unroll
    for (int l = 0; l < 16; ++l) acc[l] = 0.f;
    const float4* x4 = reinterpret_cast<const float4*>(x);
    const float4* q4 = reinterpret_cast<const float4*>(q);
    uint32_t i = 0;
    for (; i + 2 <= nb; i += 2) {
        float4 a[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) a[c] = __ldg(x4 + 4 * i + c);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const float4 p = q4[4 * i + c];
            const int l = (c & 3) * 4;
            acc[l + 0] = sq_step(acc[l + 0], p.x - a[c].x, FUSED);
            acc[l + 1] = sq_step(acc[l + 1], p.y - a[c].y, FUSED);
            acc[l + 2] = sq_step(acc[l + 2], p.z - a[c].z, FUSED);
            acc[l + 3] = sq_step(acc[l + 3], p.w - a[c].w, FUSED);
        }
    }
    if (i < nb) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const float4 a = __ldg(x4 + 4 * i + c);
            const float4 p = q4[4 * i + c];
            const int l = c * 4;
            acc[l + 0] = sq_step(acc[l + 0], p.x - a.x, FUSED);
            acc[l + 1] = sq_step(acc[l + 1], p.y - a.y, FUSED);
            acc[l + 2] = sq_step(acc[l + 2], p.z - a.z, FUSED);
            acc[l + 3] = sq_step(acc[l + 3], p.w - a.w, FUSED);
        }
    }
    float s = acc[0];
#pragma unroll
    for (int l = 1; l < 16; ++l) s = __fadd_rn(s, acc[l]);
    return s;
}

// Two lanes per row (lane parity p owns accumulators 8p..8p+7, i.e. float4 #2p and
// #2p+1 of every 16-element block); all of a lane's loads for its half row are
// issued before the accumulation, so 16 rows of a warp cost one memory round trip.
template <bool FUSED, int NB>
__device__ __forceinline__ float l2_pair16(const float* __restrict__ q, const float* __restrict__ x, int p) {
    const float4* x4 = reinterpret_cast<const float4*>(x);
    const float4* q4 = reinterpret_cast<const float4*>(q);
    float4 a[2 * NB];
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        a[2 * i] = __ldg(x4 + 4 * i + 2 * p);
        a[2 * i + 1] = __ldg(x4 + 4 * i + 2 * p + 1);
    }
    float acc[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) acc[l] = 0.f;
#pragma unroll
    for (int i = 0; i < NB; ++i) {
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const float4 qq = q4[4 * i + 2 * p + c];
            const float4 xx = a[2 * i + c];
            acc[4 * c + 0] = sq_step(acc[4 * c + 0], qq.x - xx.x, FUSED);
            acc[4 * c + 1] = sq_step(acc[4 * c + 1], qq.y - xx.y, FUSED);
            acc[4 * c + 2] = sq_step(acc[4 * c + 2], qq.z - xx.z, FUSED);
            acc[4 * c + 3] = sq_step(acc[4 * c + 3], qq.w - xx.w, FUSED);
        }
    }
    // TmpRes[0] + ... + TmpRes[15] left to right: the even lane owns 0..7.
    float hi[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) hi[l] = __shfl_down_sync(0xFFFFFFFFu, acc[l], 1);
    float s = acc[0];
#pragma unroll
    for (int l = 1; l < 8; ++l) s = __fadd_rn(s, acc[l]);
#pragma unroll
    for (int l = 0; l < 8; ++l) s = __fadd_rn(s, hi[l]);
    return s;  // valid in the even lane
}

template <bool FUSED, int NB>
__device__ __forceinline__ void warp_l2_pairs(const DevView& v, const float* q, const uint32_t* ids, uint32_t cnt,
                                              float* dout) {
    const int lane = threadIdx.x & 31, p = lane & 1;
    for (uint32_t r = 0; r < cnt; r += 16) {
        const uint32_t t = r + (lane >> 1);
        const uint32_t id = ids[t < cnt ? t : r];
        const float d = l2_pair16<FUSED, NB>(q, v.vec + (size_t)id * v.dim, p);
        if (p == 0 && t < cnt) dout[t] = d;
    }
}

// Distances of q to cnt (<= 32) stored vectors ids[0..cnt) -> dout[0..cnt).
// dims 96/128/256 with the 16-lane order: two lanes per row (l2_pair16);
// other multiples of 16: one row per lane; other dims or orders: l2_thread.
template <bool FUSED>
__device__ __forceinline__ void warp_l2_list(const DevView& v, const float* q, const uint32_t* ids, uint32_t cnt,
                                             float* dout) {
    const int lane = threadIdx.x & 31;
    if (v.lanes == 16 && v.nb == 8 && v.dim == 128) {
        warp_l2_pairs<FUSED, 8>(v, q, ids, cnt, dout);
    } else if (v.lanes == 16 && v.nb == 6 && v.dim == 96) {
        warp_l2_pairs<FUSED, 6>(v, q, ids, cnt, dout);
    } else if (v.lanes == 16 && v.nb == 16 && v.dim == 256) {
        warp_l2_pairs<FUSED, 16>(v, q, ids, cnt, dout);
    } else {
        for (uint32_t t = lane; t < cnt; t += 32) {
            const float* x = v.vec + (size_t)ids[t] * v.dim;
            dout[t] = (v.lanes == 16 && v.dim % 16 == 0) ? l2_row16<FUSED>(q, x, v.nb)
                                                         : l2_thread(q, x, v.dim, v.lanes, v.fused);
        }
    }
    __syncwarp();
}

struct WarpSmem {
    float* q;
    float* td;       // beam distances (ascending)
    uint32_t* ti;    // beam ids | kExpanded
    float* xd;       // merge scratch
    uint32_t* xi;
    uint32_t* vis;   // visited cache
    float* nd;       // neighbour distances
    uint32_t* ni;    // neighbour ids
    uint32_t* apos;  // accepted insertion points
    int* q8;         // INT8 beam: the query as packed int8 words (dim / 4)
    float4* qm;      // (s_q^2 sum q8^2, s_q, ||q - s_q q8||, 0)
};

__host__ __device__ inline size_t warp_smem_bytes(uint32_t dim, uint32_t efc, uint32_t vc) {
    // multiple of 16 for dim % 4 == 0 and efc % 32 == 0 (q is read as float4)
    return (size_t)dim * 4 + (((size_t)dim + 15) & ~(size_t)15) + 16 + (size_t)(efc + 32) * 8 + (size_t)vc * 4 +
           32 * 12 + 16;
}

// q | q8 (dim bytes, padded to 16) | qm (16 bytes) | td | ti | vis | nd | ni | apos
__device__ inline WarpSmem carve(char* base, uint32_t dim, uint32_t efc, uint32_t vc) {
    WarpSmem s;
    s.q = (float*)base;
    base += (size_t)dim * 4;
    s.q8 = (int*)base;
    base += ((size_t)dim + 15) & ~(size_t)15;
    s.qm = (float4*)base;
    base += 16;
    s.td = (float*)base;
    base += (size_t)(efc + 32) * 4;
    s.ti = (uint32_t*)base;
    base += (size_t)(efc + 32) * 4;
    s.xd = nullptr;
    s.xi = nullptr;
    s.vis = (uint32_t*)base;
    base += (size_t)vc * 4;
    s.nd = (float*)base;
    base += 32 * 4;
    s.ni = (uint32_t*)base;
    base += 32 * 4;
    s.apos = (uint32_t*)base;
    return s;
}

// The INT8 query words and scalars that follow a warp's q (carve's layout).
__device__ __forceinline__ const int* i8_q_words(const float* q, uint32_t dim) {
    return reinterpret_cast<const int*>(q + dim);
}
__device__ __forceinline__ const float4* i8_q_meta(const float* q, uint32_t dim) {
    return reinterpret_cast<const float4*>(reinterpret_cast<const char*>(q + dim) + ((dim + 15) & ~15u));
}

// Words of the link row of c at `level`, loaded unconditionally (no dependence on
// the count): lane j gets word j (j < row width), lane 0 also word 32 (rows of 33
// words, maxM0 = 32).  All loads stay inside the row.
__device__ __forceinline__ void load_row(const DevView& v, uint32_t c, int level, uint32_t& w0, uint32_t& w1) {
    const int lane = threadIdx.x & 31;
    const uint32_t W = level == 0 ? v.W0 : v.WU;
    const uint32_t* row = links_of(v, c, level);
    w0 = (uint32_t)lane < W ? __ldg(row + lane) : 0u;
    w1 = (lane == 0 && W > 32) ? __ldg(row + 32) : 0u;
}

// First index in td[0..n) with td[i] > x.
__device__ __forceinline__ uint32_t upper_bound(const float* td, uint32_t n, float x) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (td[mid] > x) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// BF16 rows (mixed-precision search): vec_bf16[n][dim] holds round-to-nearest
// copies of the FP32 rows.  These distances rank candidates only; every
// accept/reject decision is re-made against the FP32 rows (search_bc.cu).
// ---------------------------------------------------------------------------

__device__ __forceinline__ float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

// Two lanes per row, NB 16-element blocks: lane parity p reads bytes
// [64p, 64p+64) of every 128-byte chunk, i.e. elements 32c + 16p .. 32c + 16p + 15
// of chunk c; accumulation order is free (FP32, fused).
template <int NB>
__device__ __forceinline__ float bf16_pair(const float* __restrict__ q, const uint16_t* __restrict__ x, int p) {
    const uint4* x4 = reinterpret_cast<const uint4*>(x);
    constexpr int NC = NB / 2;  // 32-element chunks
    uint4 a[2 * NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        a[2 * c] = __ldg(x4 + 4 * c + 2 * p);
        a[2 * c + 1] = __ldg(x4 + 4 * c + 2 * p + 1);
    }
    float s0 = 0.f, s1 = 0.f;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint4 w = a[2 * c + h];
            const float* qq = q + 32 * c + 16 * p + 8 * h;
            float t;
            t = qq[0] - bf16_lo(w.x); s0 = fmaf(t, t, s0);
            t = qq[1] - bf16_hi(w.x); s1 = fmaf(t, t, s1);
            t = qq[2] - bf16_lo(w.y); s0 = fmaf(t, t, s0);
            t = qq[3] - bf16_hi(w.y); s1 = fmaf(t, t, s1);
            t = qq[4] - bf16_lo(w.z); s0 = fmaf(t, t, s0);
            t = qq[5] - bf16_hi(w.z); s1 = fmaf(t, t, s1);
            t = qq[6] - bf16_lo(w.w); s0 = fmaf(t, t, s0);
            t = qq[7] - bf16_hi(w.w); s1 = fmaf(t, t, s1);
        }
    }
    float s = s0 + s1;
    return s + __shfl_xor_sync(0xFFFFFFFFu, s, 1);  // both lanes of the pair
}

// Any dim (one lane per row, scalar), for dims not a multiple of 32.
__device__ __forceinline__ float bf16_thread(const float* __restrict__ q, const uint16_t* __restrict__ x, uint32_t d) {
    float s = 0.f;
    for (uint32_t e = 0; e < d; ++e) {
        float t = q[e] - __uint_as_float((uint32_t)x[e] << 16);
        s = fmaf(t, t, s);
    }
    return s;
}

// ---------------------------------------------------------------------------
// INT8 rows (INT8 beam): x ~ s c, c in [-127, 127]; the query is quantised the
// same way (s_q, q8) by the warp that searches it.  The approximate squared
// distance ||s_q q8 - s c||^2 = s_q^2 sum q8^2 + s^2 sum c^2 - 2 s_q s (q8 . c)
// takes integer dot products (dp4a) only; it ranks the beam, nothing else.
// ---------------------------------------------------------------------------

// The warp quantises s.q (FP32, dim floats) into s.q8 / s.qm.
__device__ __forceinline__ void i8_prep_query(const WarpSmem& s, uint32_t dim) {
    const int lane = threadIdx.x & 31;
    float mx = 0.f;
    for (uint32_t j = lane; j < dim; j += 32) mx = fmaxf(mx, fabsf(s.q[j]));
    for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    const float sc = mx > 0.f ? mx / 127.f : 1.f;
    int8_t* q8b = reinterpret_cast<int8_t*>(s.q8);
    double e2 = 0.0;
    int c2 = 0;
    for (uint32_t j = lane; j < dim; j += 32) {
        const int c = max(-127, min(127, __float2int_rn(s.q[j] / sc)));
        q8b[j] = (int8_t)c;
        const double dlt = (double)s.q[j] - (double)sc * (double)c;
        e2 += dlt * dlt;
        c2 += c * c;
    }
    for (int o = 16; o; o >>= 1) {
        e2 += __shfl_xor_sync(0xFFFFFFFFu, e2, o);
        c2 += __shfl_xor_sync(0xFFFFFFFFu, c2, o);
    }
    if (lane == 0) *s.qm = make_float4(sc * sc * (float)c2, sc, __double2float_ru(sqrt(e2)), 0.f);
    __syncwarp();
}

// NW 16-byte words of one row (dim = 16 NW), all loaded before the dot products.
template <int NW>
__device__ __forceinline__ float i8_row(const int* __restrict__ q8, float4 qm, const int8_t* __restrict__ x,
                                        float4 xm) {
    const int4* x4 = reinterpret_cast<const int4*>(x);
    int4 a[NW];
#pragma unroll
    for (int c = 0; c < NW; ++c) a[c] = __ldg(x4 + c);
    int dot = 0;
#pragma unroll
    for (int c = 0; c < NW; ++c) {
        dot = __dp4a(a[c].x, q8[4 * c + 0], dot);
        dot = __dp4a(a[c].y, q8[4 * c + 1], dot);
        dot = __dp4a(a[c].z, q8[4 * c + 2], dot);
        dot = __dp4a(a[c].w, q8[4 * c + 3], dot);
    }
    return qm.x + xm.x * xm.x * xm.z - 2.f * qm.y * xm.x * (float)dot;
}

template <int NW>
__device__ __forceinline__ void warp_i8_rows(const DevView& v, const int* q8, float4 qm, const uint32_t* ids,
                                             uint32_t cnt, float* dout) {
    const int lane = threadIdx.x & 31;
    for (uint32_t r = 0; r < cnt; r += 32) {
        const uint32_t t = r + lane;
        const uint32_t id = ids[t < cnt ? t : r];
        const float d = i8_row<NW>(q8, qm, v.vec_i8 + (size_t)id * v.dim, __ldg(v.i8_meta + id));
        if (t < cnt) dout[t] = d;
    }
}

__device__ __forceinline__ void warp_i8_list(const DevView& v, const int* q8, float4 qm, const uint32_t* ids,
                                             uint32_t cnt, float* dout) {
    // dim = 16 NW exactly (the precision setter allows multiples of 16 up to 256)
    switch (v.dim >> 4) {
#define HRNN_I8_CASE(W) \
    case W: warp_i8_rows<W>(v, q8, qm, ids, cnt, dout); break;
        HRNN_I8_CASE(1) HRNN_I8_CASE(2) HRNN_I8_CASE(3) HRNN_I8_CASE(4) HRNN_I8_CASE(5) HRNN_I8_CASE(6)
        HRNN_I8_CASE(7) HRNN_I8_CASE(8) HRNN_I8_CASE(9) HRNN_I8_CASE(10) HRNN_I8_CASE(11) HRNN_I8_CASE(12)
        HRNN_I8_CASE(13) HRNN_I8_CASE(14) HRNN_I8_CASE(15) HRNN_I8_CASE(16)
#undef HRNN_I8_CASE
        default: break;
    }
    __syncwarp();
}

// Cooperative INT8 row reads.  In round i of a block of eight rounds, lane
// (g, s) = (lane >> 3, lane & 7) reads bytes 16 s .. 16 s + 15 of row 4 i + g of a
// block of 32 rows, so one 16-byte load per lane covers four whole rows (one
// 128-byte line each) instead of 32 scattered ones; lanes with s >= NB (rows
// narrower than 128 bytes) read nothing.
template <int NB>
__device__ __forceinline__ int4 coop_i8_load(const int8_t* vec, uint32_t id) {
    const int s = threadIdx.x & 7;
    return s < NB ? __ldg(reinterpret_cast<const int4*>(vec + (size_t)id * (NB * 16)) + s) : make_int4(0, 0, 0, 0);
}

__device__ __forceinline__ int dp4a4(int4 a, int4 b) {
    return __dp4a(a.x, b.x, __dp4a(a.y, b.y, __dp4a(a.z, b.z, __dp4a(a.w, b.w, 0))));
}

// The row of a block whose whole dot product coop_sum8 leaves in this lane.
__device__ __forceinline__ uint32_t coop_row() { return 4 * (threadIdx.x & 7) + ((threadIdx.x >> 3) & 3); }

// Folds the eight partial dot products p[i] (round i) of the lanes of a group of
// eight so that lane (g, s) ends with the sum over the group of p[s] -- the whole
// dot product of row 4 s + g.  Three butterfly steps, each swapping half of the
// values still held: 4 + 2 + 1 shuffles for eight rows.
__device__ __forceinline__ int coop_sum8(const int (&p)[8]) {
    const int s = threadIdx.x & 7;
    const bool b2 = s & 4, b1 = s & 2, b0 = s & 1;
    int w[4], x[2];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int send = b2 ? p[k] : p[k + 4], keep = b2 ? p[k + 4] : p[k];
        w[k] = keep + __shfl_xor_sync(0xFFFFFFFFu, send, 4);
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int send = b1 ? w[k] : w[k + 2], keep = b1 ? w[k + 2] : w[k];
        x[k] = keep + __shfl_xor_sync(0xFFFFFFFFu, send, 2);
    }
    const int send = b0 ? x[0] : x[1], keep = b0 ? x[1] : x[0];
    return keep + __shfl_xor_sync(0xFFFFFFFFu, send, 1);
}

// This lane's INT8 query words for the cooperative reads (bytes 16 s .. 16 s + 15).
template <int NB>
__device__ __forceinline__ int4 coop_q_words(const int* q8) {
    const int s = threadIdx.x & 7;
    return s < NB ? make_int4(q8[4 * s], q8[4 * s + 1], q8[4 * s + 2], q8[4 * s + 3]) : make_int4(0, 0, 0, 0);
}

// One row scored by every lane (the entry point of a search).
__device__ __forceinline__ float i8_one(const DevView& v, const float* q, uint32_t id) {
    const int* q8 = i8_q_words(q, v.dim);
    const float4 qm = *i8_q_meta(q, v.dim);
    const int8_t* x = v.vec_i8 + (size_t)id * v.dim;
    const float4 xm = __ldg(v.i8_meta + id);
    switch (v.dim >> 4) {
#define HRNN_I8_ONE(W) \
    case W: return i8_row<W>(q8, qm, x, xm);
        HRNN_I8_ONE(1) HRNN_I8_ONE(2) HRNN_I8_ONE(3) HRNN_I8_ONE(4) HRNN_I8_ONE(5) HRNN_I8_ONE(6)
        HRNN_I8_ONE(7) HRNN_I8_ONE(8) HRNN_I8_ONE(9) HRNN_I8_ONE(10) HRNN_I8_ONE(11) HRNN_I8_ONE(12)
        HRNN_I8_ONE(13) HRNN_I8_ONE(14) HRNN_I8_ONE(15) HRNN_I8_ONE(16)
#undef HRNN_I8_ONE
        default: return 0.f;
    }
}

template <int NB>
__device__ __forceinline__ void warp_bf16_pairs(const DevView& v, const float* q, const uint32_t* ids, uint32_t cnt,
                                                float* dout) {
    const int lane = threadIdx.x & 31, p = lane & 1;
    for (uint32_t r = 0; r < cnt; r += 16) {
        const uint32_t t = r + (lane >> 1);
        const uint32_t id = ids[t < cnt ? t : r];
        const float d = bf16_pair<NB>(q, v.vec_bf16 + (size_t)id * v.dim, p);
        if (p == 0 && t < cnt) dout[t] = d;
    }
}

// Distance modes: 0 = exact FP32 unfused, 1 = exact FP32 fused, 2 = BF16 rows.
template <int DM>
__device__ __forceinline__ void warp_dist_list(const DevView& v, const float* q, const uint32_t* ids, uint32_t cnt,
                                               float* dout) {
    if constexpr (DM == 3) {
        // q is the warp's s.q; its INT8 copy and (s_q^2 sum q8^2, s_q, e_q) follow it
        warp_i8_list(v, i8_q_words(q, v.dim), *i8_q_meta(q, v.dim), ids, cnt, dout);
    } else if constexpr (DM < 2) {
        warp_l2_list<DM == 1>(v, q, ids, cnt, dout);
    } else {
        const int lane = threadIdx.x & 31;
        if (v.dim == 128) warp_bf16_pairs<8>(v, q, ids, cnt, dout);
        else if (v.dim == 96) warp_bf16_pairs<6>(v, q, ids, cnt, dout);
        else if (v.dim == 256) warp_bf16_pairs<16>(v, q, ids, cnt, dout);
        else
            for (uint32_t t = lane; t < cnt; t += 32) dout[t] = bf16_thread(q, v.vec_bf16 + (size_t)ids[t] * v.dim, v.dim);
        __syncwarp();
    }
}

template <int DM>
__device__ __forceinline__ float warp_dist_one(const DevView& v, const float* q, uint32_t id) {
    if constexpr (DM < 2) {
        return warp_l2_one<DM == 1>(v, q, id);
    } else if constexpr (DM == 3) {
        return i8_one(v, q, id);
    } else {
        return bf16_thread(q, v.vec_bf16 + (size_t)id * v.dim, v.dim);
    }
}

// Greedy descent over levels top..stop+1 (hrnn.h:1992-2013, 1438-1464): per level,
// move to the first strict improvement of the running minimum in list order
// until a whole list brings none.  cur/curd are updated in every lane.
template <int DM>
__device__ void greedy_descent(const DevView& v, WarpSmem& s, int top, int stop, uint32_t& cur, float& curd,
                               unsigned long long& c_dist) {
    const int lane = threadIdx.x & 31;
    for (int level = top; level > stop; --level) {
        bool changed = true;
        while (changed) {
            changed = false;
            const uint32_t* blk = links_of(v, cur, level);
            uint32_t size = blk[0] & 0xFFFFu;
            float bestd = curd;
            uint32_t best = cur;
            for (uint32_t base = 0; base < size; base += 32) {
                uint32_t cnt = min(32u, size - base);
                if ((uint32_t)lane < cnt) s.ni[lane] = blk[1 + base + lane];
                __syncwarp();
                warp_dist_list<DM>(v, s.q, s.ni, cnt, s.nd);
                c_dist += cnt;
                float d = (uint32_t)lane < cnt ? s.nd[lane] : FLT_MAX;
                float mn = d;
                for (int o = 16; o; o >>= 1) mn = fminf(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, o));
                uint32_t hit = __ballot_sync(0xFFFFFFFFu, (uint32_t)lane < cnt && d == mn);
                if (mn < bestd) {
                    bestd = mn;
                    best = s.ni[__ffs(hit) - 1];
                    changed = true;
                }
                __syncwarp();
            }
            cur = best;
            curd = bestd;
        }
    }
}

// Inserts cnt (<= 32) scored neighbours (nd[i], ni[i]) into the beam: neighbour j
// is accepted iff fewer than EF elements of (beam + accepted earlier neighbours of
// this batch) are <= d_j, and not already in the beam; the beam stays sorted and
// is cut to EF; cursor moves back to the first inserted position.
//
// A neighbour no closer than the last entry of a full beam can be dropped before
// the rest: it would land at position EF, and it only counts against neighbours
// that are no closer than itself.  The accepted ones are ranked by (distance,
// lane), which orders their insertion points too, so apos[] is sorted and the
// shift of a beam entry is a binary search over it.
__device__ __forceinline__ void beam_insert(WarpSmem& s, const float* nd, const uint32_t* ni, uint32_t cnt,
                                            uint32_t EF, uint32_t& tsize, uint32_t& cursor) {
    const int lane = threadIdx.x & 31;
    float d = FLT_MAX;
    uint32_t id = kInvalid, pos = 0;
    bool ok = false;
    if ((uint32_t)lane < cnt) {
        d = nd[lane];
        id = ni[lane];
        ok = !(tsize >= EF && d >= s.td[EF - 1]);
    }
    if (!__ballot_sync(0xFFFFFFFFu, ok)) return;
    if (ok) {
        pos = upper_bound(s.td, tsize, d);
        for (int k = (int)pos - 1; k >= 0 && s.td[k] == d; --k)
            if ((s.ti[k] & kIdMask) == id) {
                ok = false;
                break;
            }
    }
    const uint32_t okb = __ballot_sync(0xFFFFFFFFu, ok);
    if (!okb) return;
    uint32_t cp = 0;
    for (uint32_t m = okb; m; m &= m - 1) {
        const int i = __ffs(m) - 1;
        const float di = __shfl_sync(0xFFFFFFFFu, d, i);
        if (i < lane && di <= d) cp++;
    }
    const bool acc = ok && (pos + cp < EF);
    const uint32_t ab = __ballot_sync(0xFFFFFFFFu, acc);
    if (!ab) return;
    const uint32_t na = __popc(ab);
    uint32_t before = 0;
    for (uint32_t m = ab; m; m &= m - 1) {
        const int i = __ffs(m) - 1;
        const float di = __shfl_sync(0xFFFFFFFFu, d, i);
        if (di < d || (di == d && i < lane)) before++;
    }
    if (acc) s.apos[before] = pos;
    __syncwarp();
    const uint32_t lo = s.apos[0], amax = s.apos[na - 1];
    const uint32_t newsize = min(tsize + na, EF);
    // In-place merge: existing entries at or after lo move right by the number
    // of accepted neighbours inserted at or before them (at most 32), so the
    // beam is shifted block by block from the right; every block is read
    // before any lane writes, and its targets lie in itself or in blocks to
    // its right that were already moved.
    if (tsize > lo) {
        for (int b = (int)lo + (int)(((tsize - lo - 1) / 32) * 32); b >= (int)lo; b -= 32) {
            const uint32_t k = (uint32_t)b + lane;
            float dk = 0.f;
            uint32_t ik = 0, np = 0xFFFFFFFFu;
            if (k < tsize) {
                dk = s.td[k];
                ik = s.ti[k];
                uint32_t sh = na;
                if (k < amax) {  // number of insertion points <= k
                    uint32_t a = 0, e = na - 1;
                    while (a < e) {
                        const uint32_t mid = (a + e) >> 1;
                        if (s.apos[mid] <= k) a = mid + 1;
                        else e = mid;
                    }
                    sh = a;
                }
                np = k + sh;
            }
            __syncwarp();
            if (np < newsize) {
                s.td[np] = dk;
                s.ti[np] = ik;
            }
            __syncwarp();
        }
    }
    const uint32_t npos = pos + before;
    if (acc && npos < newsize) {
        s.td[npos] = d;
        s.ti[npos] = id;
    }
    uint32_t mnp = (acc && npos < newsize) ? npos : 0xFFFFFFFFu;
    for (int o = 16; o; o >>= 1) mnp = min(mnp, __shfl_xor_sync(0xFFFFFFFFu, mnp, o));
    tsize = newsize;
    cursor = min(cursor, mnp);
    __syncwarp();
}

// Best-first search of one layer from (ep, epd) with beam size EF (<= efc).
// On return the beam s.td/s.ti[0..tsize) holds the EF nearest found, ascending
// (ids still carry the expanded flag).  vc: visited-cache slots (power of two).
template <int DM>
__device__ uint32_t beam_search(const DevView& v, WarpSmem& s, uint32_t ep, float epd, uint32_t EF, int level,
                                uint32_t vc, unsigned long long& c_dist, unsigned long long& c_exp) {
    const int lane = threadIdx.x & 31;
    for (uint32_t i = lane; i < vc; i += 32) s.vis[i] = kInvalid;
    __syncwarp();
    // Rows of at most 33 words (maxM0 <= 32) are read whole by the warp in one go.
    const bool short_rows = (level == 0 ? v.W0 : v.WU) <= 33;
    uint32_t tsize = 1, cursor = 0;
    if (lane == 0) {
        s.td[0] = epd;
        s.ti[0] = ep;
        s.vis[hash32(ep) & (vc - 1)] = ep;
    }
    __syncwarp();
    for (;;) {
        int found = -1;
        for (uint32_t b = cursor; b < tsize; b += 32) {
            uint32_t idx = b + lane;
            bool u = idx < tsize && !(s.ti[idx] & kExpanded);
            uint32_t bal = __ballot_sync(0xFFFFFFFFu, u);
            if (bal) {
                found = (int)(b + __ffs(bal) - 1);
                break;
            }
        }
        if (found < 0) break;
        cursor = (uint32_t)found + 1;
        const uint32_t c = s.ti[found] & kIdMask;
        __syncwarp();
        if (lane == 0) s.ti[found] |= kExpanded;
        c_exp++;
        // Links of c: one unconditional load of the row's words (no dependence on
        // the count word).
        uint32_t row0 = 0, row1 = 0;
        if (short_rows) load_row(v, c, level, row0, row1);
        const uint32_t* adj = links_of(v, c, level);
        if (!short_rows) row0 = adj[0];
        const uint32_t size = __shfl_sync(0xFFFFFFFFu, row0, 0) & 0xFFFFu;
        for (uint32_t base = 0; base < size; base += 32) {
            uint32_t j = base + lane;
            uint32_t nid;
            if (short_rows) {  // id j is word j + 1 of the row
                const uint32_t a = __shfl_sync(0xFFFFFFFFu, row0, (lane + 1) & 31);
                const uint32_t b = __shfl_sync(0xFFFFFFFFu, row1, 0);
                nid = j < size ? (lane < 31 ? a : b) : kInvalid;
            } else {
                nid = j < size ? adj[1 + j] : kInvalid;
            }
            uint32_t slot = hash32(nid) & (vc - 1);
            bool fresh = j < size && s.vis[slot] != nid;
            __syncwarp();
            uint32_t fb = __ballot_sync(0xFFFFFFFFu, fresh);
            uint32_t cnt = __popc(fb);
            if (fresh) {
                s.ni[__popc(fb & lanemask_lt())] = nid;
                s.vis[slot] = nid;
            }
            __syncwarp();
            if (cnt == 0) continue;
            warp_dist_list<DM>(v, s.q, s.ni, cnt, s.nd);
            c_dist += cnt;
            beam_insert(s, s.nd, s.ni, cnt, EF, tsize, cursor);
        }
    }
    return tsize;
}

}  // namespace hrnn
