// Streaming verification of the INT8 search form (threshold <= 1, dims 96 and
// 128): phase B + C of searchRknn (hrnn.h:2021-2070) without a candidate table.
//
// Every posting of the proxies' reverse-list prefixes (rank < K') is verified
// where it is read.  The postings are cut into chunks of kChunk (a proxy's prefix
// into several when it is long), and persistent warps take chunks from a counter,
// so one query with a proxy of a very long reverse list is spread over many warps
// instead of holding one.  Per posting the INT8 screen first (rows read by eight
// lanes each, four rows per load instruction, dp4a against the query); the
// few rows it cannot decide in exact FP32 (the reference's order, a half-warp per
// row) and, inside kTieUlps of the radius, in FP64.  An owner listed by several
// proxies is verified once per listing -- the same decision each time.
//
// Accepted ids go to the query's slice of the result buffer (as many slots as the
// query has postings, so it cannot overflow); a finishing pass sorts each query's
// ids, drops repeats and writes the labels in ascending internal-id order
// (hrnn.h:2055).  With every count >= 1 passing the threshold (hrnn.h:2043-2052)
// the candidate set and every decision are the CTA table kernel's, so are the
// answers.  A query with more than kFinCap acceptances (repeats included) is
// listed for the overflow pass, which answers it from scratch.
#include <algorithm>
#include <cfloat>
#include <cstdlib>
#include <type_traits>

#include "beam.cuh"
#include "index.hpp"
#include "verify_stream.hpp"

namespace hrnn {

namespace {

constexpr uint32_t kChunk = 256;     // postings per work item
constexpr uint32_t kFinCap = 1024;   // acceptances a query's finishing warp sorts in shared memory
constexpr uint32_t kBigCap = 16384;  // ... and a finishing block (64 KB of shared memory)
constexpr float kTieUlpsS = 16.f;    // FP64 re-decision band around the radius, in ulps of kd

// The INT8 screen of one row: 1 accept, 0 reject, -1 undecided.
// |sqrt(d) - sqrt(D)| <= e_q + e_x with D = ||s_q q8 - s c||^2 evaluated in FP32
// within 8 ulps of (sqrt(s_q^2 sum q8^2) + s sqrt(sum c^2))^2; rho covers the
// reference's own FP32 sum and this bound's roundings.
__device__ __forceinline__ int i8_decide(float D, float kd, float4 qv, float4 xm, uint32_t dim) {
    if (kd == FLT_MAX) return 1;
    const float rq = sqrtf(qv.x), rx = xm.x * sqrtf(xm.z);
    const float ef = 8.f * 5.9604645e-8f * (rq + rx) * (rq + rx);
    const float e = qv.z + xm.y;
    const float rho = (4.f * dim + 64.f) * 5.9604645e-8f;
    const float hi = sqrtf(D + ef) * (1.f + rho) + e;
    const float lo = fmaxf(0.f, sqrtf(fmaxf(0.f, D - ef)) * (1.f - rho) - e);
    const float U = hi * hi * (1.f + rho), L = lo * lo * (1.f - rho);
    return U < kd ? 1 : (L > kd ? 0 : -1);
}

// The INT8 copy of every query (as i8_prep_query): int8 rows qq[nq][dim] and
// (s_q^2 sum q8^2, s_q, ||q - s_q q8||, 0) per query.  One warp per query.
__global__ void k_quantize_queries(const float* __restrict__ Q, uint32_t nq, uint32_t dim,
                                   int8_t* __restrict__ qq, float4* __restrict__ qmeta) {
    const uint32_t qi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (qi >= nq) return;
    const float* q = Q + (size_t)qi * dim;
    float mx = 0.f;
    for (uint32_t j = lane; j < dim; j += 32) mx = fmaxf(mx, fabsf(q[j]));
    for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    const float sc = mx > 0.f ? mx / 127.f : 1.f;
    double e2 = 0.0;
    int c2 = 0;
    for (uint32_t j = lane; j < dim; j += 32) {
        const int c = max(-127, min(127, __float2int_rn(q[j] / sc)));
        qq[(size_t)qi * dim + j] = (int8_t)c;
        const double dlt = (double)q[j] - (double)sc * (double)c;
        e2 += dlt * dlt;
        c2 += c * c;
    }
    for (int o = 16; o; o >>= 1) {
        e2 += __shfl_xor_sync(0xFFFFFFFFu, e2, o);
        c2 += __shfl_xor_sync(0xFFFFFFFFu, c2, o);
    }
    if (lane == 0) qmeta[qi] = make_float4(sc * sc * (float)c2, sc, __double2float_ru(sqrt(e2)), 0.f);
}

// meta[i].w = kdist(i, k-1) of this call, next to the row's scale and error
// terms, so the screen reads one 16-byte record per candidate.
__global__ void k_meta_radius(const float* __restrict__ kcol, uint32_t n, float4* __restrict__ meta) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) meta[i].w = kcol[i];
}

// Chunks per (query, proxy) prefix.
__global__ void k_chunk_count(const uint32_t* __restrict__ plen, size_t npairs, uint32_t* __restrict__ cnt) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < npairs) cnt[t] = (plen[t] + kChunk - 1) / kChunk;
}

// Work items: (pair << 32) | first posting of the chunk.
__global__ void k_chunk_fill(const uint32_t* __restrict__ cnt, const uint64_t* __restrict__ coff, size_t npairs,
                             uint64_t* __restrict__ chunks) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npairs) return;
    const uint32_t c = cnt[t];
    for (uint32_t j = 0; j < c; ++j) chunks[coff[t] + j] = ((uint64_t)t << 32) | (j * kChunk);
}

// Appends the ids of the lanes with `a` set to query qi's slice of the result
// buffer (counted in acc_cnt).  A slice shorter than the query's postings (a
// captured plan's bounded staging) takes what fits; the finishing pass sends a
// query whose count passed its slice to the overflow pass.
__device__ __forceinline__ void stream_accept(bool a, uint32_t id, uint32_t qi, const uint64_t* res_off,
                                              uint32_t* acc_cnt, uint64_t* resbuf) {
    const uint32_t ab = __ballot_sync(0xFFFFFFFFu, a);
    if (!ab) return;
    const int lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(&acc_cnt[qi], (uint32_t)__popc(ab));
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    if (a) {
        const uint64_t pos = res_off[qi] + base + __popc(ab & ((1u << lane) - 1u));
        if (pos < res_off[qi + 1]) resbuf[pos] = id;
    }
}

// Counters of one warp (summed into SearchCounters at the end).
struct StreamCount {
    unsigned long long lowp = 0, fp32 = 0, fp64 = 0, flip = 0;
};

// The rows the INT8 screen left undecided (lanes with dec < 0): the BF16 screen
// (two lanes per row), then exact FP32 in the reference's order (a half-warp per
// row) and FP64 inside the tie band.  Kept out of line: it is rare, and its
// registers would otherwise weigh on the streaming loop.
template <bool FUSED, int NB>
__device__ __noinline__ void stream_undecided(const DevView& v, const float* __restrict__ Q, uint32_t qi, int dec,
                                              uint32_t id, float* q, uint32_t* st, uint32_t& f32_q,
                                              const float* __restrict__ kcol, uint32_t kidx,
                                              const uint64_t* __restrict__ res_off, uint32_t* __restrict__ acc_cnt,
                                              uint64_t* __restrict__ resbuf, StreamCount& cn) {
    constexpr uint32_t dim = NB * 16;
    const int lane = threadIdx.x & 31;
    const uint32_t und = __ballot_sync(0xFFFFFFFFu, dec < 0);
    if (f32_q != qi) {
        __syncwarp();
        for (uint32_t i = lane; i < dim; i += 32) q[i] = Q[(size_t)qi * dim + i];
        f32_q = qi;
    }
    __syncwarp();
    if (dec < 0) st[__popc(und & ((1u << lane) - 1u))] = id;
    __syncwarp();
    uint32_t nu = 0;
    const uint32_t nu8 = __popc(und);
    for (uint32_t r = 0; r < nu8; r += 16) {
        const int pp = lane & 1;
        const uint32_t tt = r + (lane >> 1);
        const bool lv = tt < nu8;
        const uint32_t x = st[lv ? tt : r];
        const float kx = __ldg(kcol + x);
        const float D = bf16_pair<NB>(q, v.vec_bf16 + (size_t)x * dim, pp);
        const float ex = __ldg(v.vec_err + x);
        const float rho = (4.f * dim + 64.f) * 5.9604645e-8f;
        const float sD = sqrtf(D);
        const float hi = sD * (1.f + rho) + ex, lo = fmaxf(0.f, sD * (1.f - rho) - ex);
        const float U = hi * hi * (1.f + rho), L = lo * lo * (1.f - rho);
        const int db = kx == FLT_MAX ? 1 : (U < kx ? 1 : (L > kx ? 0 : -1));
        if (lv && pp == 0 && db >= 0) cn.lowp++;
        stream_accept(lv && pp == 0 && db == 1, x, qi, res_off, acc_cnt, resbuf);
        const uint32_t u2 = __ballot_sync(0xFFFFFFFFu, lv && pp == 0 && db < 0);
        __syncwarp();  // every lane has read its row of this round
        if (lv && pp == 0 && db < 0) st[nu + __popc(u2 & ((1u << lane) - 1u))] = x;
        nu += __popc(u2);
        __syncwarp();
    }
    const int hh = lane >> 4, l16 = lane & 15;  // one row per half-warp
    for (uint32_t r = 0; r < nu; r += 2) {
        const uint32_t tt = r + hh;
        const bool lv = tt < nu;
        const uint32_t x = st[lv ? tt : r];
        const float kx = __ldg(kcol + x);
        const float d32 = l2_half16<FUSED>(q, v.vec + (size_t)x * dim, NB, l16);
        int decision = d32 <= kx;
        if (lv && l16 == 0) cn.fp32++;
        const bool tie = lv && kx != FLT_MAX && v.knn_ids && kidx < (v.knn_hdr[x] & 0xFFFFu) &&
                         fabsf(d32 - kx) <= kTieUlpsS * (nextafterf(kx, FLT_MAX) - kx);
        if (__any_sync(0xFFFFFFFFu, tie)) {
            // FP64: d(q, x) against d(x, x_k), x_k the k-th neighbour of x
            double a = 0.0, bb = 0.0;
            if (tie) {
                const uint32_t nk = v.knn_ids[(size_t)x * v.K + kidx];
                const float* xr = v.vec + (size_t)x * dim;
                const float* yr = v.vec + (size_t)nk * dim;
                for (uint32_t e2 = l16; e2 < dim; e2 += 16) {
                    const double tq = (double)q[e2] - (double)xr[e2];
                    const double ty = (double)xr[e2] - (double)yr[e2];
                    a += tq * tq;
                    bb += ty * ty;
                }
            }
            for (int o = 8; o; o >>= 1) {
                a += __shfl_xor_sync(0xFFFFFFFFu, a, o);
                bb += __shfl_xor_sync(0xFFFFFFFFu, bb, o);
            }
            if (tie) {
                const int d64 = a <= bb;
                if (l16 == 0) {
                    cn.fp64++;
                    if (d64 != decision) cn.flip++;
                }
                decision = d64;
            }
        }
        stream_accept(lv && l16 == 0 && decision == 1, x, qi, res_off, acc_cnt, resbuf);
    }
    __syncwarp();
}

// S steps of 32 postings through the INT8 screen, the loads of all S steps' rows
// issued before any dot product: 1 accept, 0 reject, -1 undecided each; meta.w
// holds kdist(p, k-1) of this call.  The rows are read cooperatively
// (coop_i8_load): eight rounds of four whole rows per load instruction per step
// instead of 32 rows touched per instruction -- the one-row-per-lane form kept
// the L1 saturated with line lookups.  cid: the owner ids of the steps (32 per
// step, shared memory); out: the id this lane decides in each step, posting
// coop_row() of the step (live[s]: whether that posting exists).  qw: this lane's
// query words (coop_q_words).
template <int NB, int S>
__device__ __forceinline__ void stream_screen_coop(const DevView& v, int4 qw, float4 qv, const uint32_t* cid,
                                                   const bool (&live)[S], uint32_t (&out)[S], int (&dec)[S]) {
    constexpr uint32_t dim = NB * 16;
    const int g = (threadIdx.x >> 3) & 3;
    const uint32_t r = coop_row();
    int4 x[S][8];
#pragma unroll
    for (int k = 0; k < S; ++k) {
        out[k] = cid[32 * k + r];
#pragma unroll
        for (int i = 0; i < 8; ++i) x[k][i] = coop_i8_load<NB>(v.vec_i8, cid[32 * k + 4 * i + g]);
    }
    float4 m[S];
#pragma unroll
    for (int k = 0; k < S; ++k) m[k] = __ldg(v.i8_meta + out[k]);
#pragma unroll
    for (int k = 0; k < S; ++k) {
        int pp[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) pp[i] = dp4a4(x[k][i], qw);
        const int dot = coop_sum8(pp);
        const float D = qv.x + m[k].x * m[k].x * m[k].z - 2.f * qv.y * m[k].x * (float)dot;
        dec[k] = live[k] ? i8_decide(D, m[k].w, qv, m[k], dim) : 0;
    }
}

// S: steps of 32 postings in flight per warp (2: more loads in flight per warp;
// 1: fewer registers, more resident warps -- the default).
template <int S>
constexpr int verify_min_blocks() {
    return S == 2 ? 2 : 4;
}

// Per-warp shared memory: FP32 query | undecided ids of a step (32) | the
// chunk's owner ids (kChunk).
__host__ __device__ constexpr size_t verify_warp_smem(uint32_t dim) {
    return (size_t)dim * 4 + 32 * 4 + kChunk * 4;
}

template <class E, bool FUSED, int NB, int S>
__global__ void __launch_bounds__(256, verify_min_blocks<S>()) k_verify_chunks(
    DevView v, const float* __restrict__ Q, uint32_t mmax, const uint32_t* __restrict__ prox,
    const uint32_t* __restrict__ plen, const uint64_t* __restrict__ res_off, const float* __restrict__ kcol,
    uint32_t kidx, const int8_t* __restrict__ qq, const float4* __restrict__ qmeta,
    const uint64_t* __restrict__ chunks, const uint64_t* __restrict__ nchunks, uint32_t* __restrict__ next,
    uint32_t* __restrict__ acc_cnt, uint64_t* __restrict__ resbuf, SearchCounters* __restrict__ ctr) {
    extern __shared__ __align__(16) char smraw[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    constexpr uint32_t dim = NB * 16;
    constexpr int kSteps = kChunk / 32;
    char* base = smraw + (size_t)w * verify_warp_smem(dim);
    float* q = (float*)base;                  // FP32 query (loaded when a row needs the exact test)
    uint32_t* st = (uint32_t*)(q + dim);      // undecided ids of a step
    uint32_t* cid = st + 32;                  // owner ids of the chunk
    const uint64_t nch = *nchunks;
    uint32_t cur_q = kInvalid, f32_q = kInvalid;
    float4 qv = make_float4(0.f, 0.f, 0.f, 0.f);
    int4 qw = make_int4(0, 0, 0, 0);  // this lane's INT8 query words (the cooperative row reads)
    unsigned long long c_post = 0, c_lowp8 = 0;  // the streaming loop's own counters stay in registers
    StreamCount cn;                              // the undecided path's
    for (;;) {
        uint64_t c = 0;
        if (lane == 0) c = atomicAdd((unsigned long long*)next, 1ull);
        c = __shfl_sync(0xFFFFFFFFu, c, 0);
        if (c >= nch) break;
        const uint64_t desc = chunks[c];
        const uint32_t t = (uint32_t)(desc >> 32), e0 = (uint32_t)desc;
        const uint32_t qi = t / mmax;
        const uint32_t len = plen[t];
        const uint32_t e1 = min(e0 + kChunk, len);
        const uint32_t p = prox[t];
        const uint64_t b = v.csr_off[p];
        const uint32_t nsteps = (e1 - e0 + 31) / 32;
        __syncwarp();  // the previous chunk's ids are no longer read
        // every owner id of the chunk in one round trip; postings past the end read
        // the proxy's own row (valid, never decided)
#pragma unroll
        for (int j = 0; j < kSteps; ++j) {
            const uint32_t e = e0 + lane + 32 * j;
            if ((uint32_t)j < ((nsteps + S - 1) / S) * S)
                cid[lane + 32 * j] = e < e1 ? (uint32_t)(((const E*)v.csr_ent)[b + e] >> v.rank_bits) : p;
        }
        if (qi != cur_q) {
            qv = qmeta[qi];
            qw = (lane & 7) < NB ? reinterpret_cast<const int4*>(qq + (size_t)qi * dim)[lane & 7]
                                 : make_int4(0, 0, 0, 0);
            cur_q = qi;
        }
        __syncwarp();
        if (lane == 0) c_post += e1 - e0;
#pragma unroll 1
        for (uint32_t j = 0; j < nsteps; j += S) {
            // this lane decides posting coop_row() of each step
            bool live[S];
            uint32_t id[S];
            int dec[S];
#pragma unroll
            for (int k = 0; k < S; ++k) live[k] = e0 + coop_row() + 32 * (j + k) < e1;
            stream_screen_coop<NB, S>(v, qw, qv, cid + 32 * j, live, id, dec);
#pragma unroll
            for (int k = 0; k < S; ++k) {
                c_lowp8 += (uint32_t)(dec[k] >= 0 && live[k]);
                stream_accept(dec[k] == 1, id[k], qi, res_off, acc_cnt, resbuf);
            }
#pragma unroll
            for (int k = 0; k < S; ++k)
                if (__any_sync(0xFFFFFFFFu, dec[k] < 0))
                    stream_undecided<FUSED, NB>(v, Q, qi, dec[k], id[k], q, st, f32_q, kcol, kidx, res_off, acc_cnt,
                                                resbuf, cn);
        }
    }
    unsigned long long c_lowp = c_lowp8 + cn.lowp, c_fp32 = cn.fp32, c_fp64 = cn.fp64, c_flip = cn.flip;
    for (int o = 16; o; o >>= 1) {
        c_lowp += __shfl_xor_sync(0xFFFFFFFFu, c_lowp, o);
        c_fp32 += __shfl_xor_sync(0xFFFFFFFFu, c_fp32, o);
        c_fp64 += __shfl_xor_sync(0xFFFFFFFFu, c_fp64, o);
        c_flip += __shfl_xor_sync(0xFFFFFFFFu, c_flip, o);
    }
    if (lane == 0) {
        atomicAdd(&ctr->n_posting, c_post);
        atomicAdd(&ctr->n_cand, c_post);
        atomicAdd(&ctr->n_verified, c_post);
        atomicAdd(&ctr->n_lowp, c_lowp);
        atomicAdd(&ctr->n_fp32, c_fp32);
        atomicAdd(&ctr->n_fp64, c_fp64);
        atomicAdd(&ctr->n_flip, c_flip);
    }
}

// One warp per query: sort the accepted ids (bitonic, shared memory), drop
// repeats, write the labels over the query's slice; queries with more than
// kFinCap acceptances are listed for k_stream_finish_big.
__global__ void __launch_bounds__(256) k_stream_finish(DevView v, uint32_t nq, const uint64_t* __restrict__ res_off,
                                                       const uint32_t* __restrict__ acc_cnt,
                                                       uint64_t* __restrict__ resbuf, uint32_t* __restrict__ res_count,
                                                       uint32_t* __restrict__ big, uint32_t* __restrict__ n_big,
                                                       SearchCounters* __restrict__ ctr,
                                                       const uint8_t* __restrict__ grp, uint8_t want) {
    __shared__ uint32_t sm[8][kFinCap];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t qi = blockIdx.x * 8 + w;
    if (qi >= nq || (grp && grp[qi] != want)) return;
    uint32_t* acc = sm[w];
    const uint32_t na = acc_cnt[qi];
    if (na > kFinCap || na > res_off[qi + 1] - res_off[qi]) {  // left to the block-wide pass
        if (lane == 0) big[atomicAdd(n_big, 1u)] = qi;
        return;
    }
    const uint64_t ro = res_off[qi];
    uint32_t P = 32;
    while (P < na) P <<= 1;
    for (uint32_t i = lane; i < P; i += 32) acc[i] = i < na ? (uint32_t)resbuf[ro + i] : kInvalid;
    __syncwarp();
    for (uint32_t k = 2; k <= P; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = lane; i < P; i += 32) {
                const uint32_t y = i ^ j;
                if (y > i) {
                    const uint32_t a0 = acc[i], a1 = acc[y];
                    if ((a0 > a1) == ((i & k) == 0)) {
                        acc[i] = a1;
                        acc[y] = a0;
                    }
                }
            }
            __syncwarp();
        }
    uint32_t nu = 0;
    for (uint32_t b0 = 0; b0 < na; b0 += 32) {
        const uint32_t i = b0 + lane;
        const bool keep = i < na && (i == 0 || acc[i] != acc[i - 1]);
        const uint32_t kb = __ballot_sync(0xFFFFFFFFu, keep);
        if (keep) resbuf[ro + nu + __popc(kb & ((1u << lane) - 1u))] = v.labels[acc[i]];
        nu += __popc(kb);
    }
    if (lane == 0) {
        res_count[qi] = nu;
        if (nu) atomicAdd(&ctr->n_result, (unsigned long long)nu);
    }
}

// Blocks per SM of one instantiation; its shared-memory attribute is set on the
// first call (outside any stream capture: stream_prepare).
// One block per listed query (blocks take them from a counter): the same with up
// to kBigCap acceptances sorted by the block in shared memory; more than that go
// to the overflow list (answered from scratch by the overflow pass).
__global__ void __launch_bounds__(1024) k_stream_finish_big(DevView v, const uint64_t* __restrict__ res_off,
                                                            const uint32_t* __restrict__ acc_cnt,
                                                            const uint32_t* __restrict__ big,
                                                            const uint32_t* __restrict__ n_big,
                                                            uint32_t* __restrict__ next, uint64_t* __restrict__ resbuf,
                                                            uint32_t* __restrict__ res_count,
                                                            uint32_t* __restrict__ ovl, uint32_t* __restrict__ n_ovl,
                                                            SearchCounters* __restrict__ ctr) {
    extern __shared__ uint32_t acc[];  // kBigCap
    __shared__ uint32_t ctl[2];
    const int tid = threadIdx.x, lane = tid & 31;
    const uint32_t nb = *n_big;
    for (;;) {
        __syncthreads();
        if (tid == 0) ctl[0] = atomicAdd(next, 1u);
        __syncthreads();
        const uint32_t b = ctl[0];
        if (b >= nb) break;
        const uint32_t qi = big[b];
        const uint32_t na = acc_cnt[qi];
        if (na > kBigCap || na > res_off[qi + 1] - res_off[qi]) {  // (or not all of them were kept)
            if (tid == 0) ovl[atomicAdd(n_ovl, 1u)] = qi;
            continue;
        }
        const uint64_t ro = res_off[qi];
        uint32_t P = 32;
        while (P < na) P <<= 1;
        for (uint32_t i = tid; i < P; i += blockDim.x) acc[i] = i < na ? (uint32_t)resbuf[ro + i] : kInvalid;
        __syncthreads();
        for (uint32_t k = 2; k <= P; k <<= 1)
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = tid; i < P; i += blockDim.x) {
                    const uint32_t y = i ^ j;
                    if (y > i) {
                        const uint32_t a0 = acc[i], a1 = acc[y];
                        if ((a0 > a1) == ((i & k) == 0)) {
                            acc[i] = a1;
                            acc[y] = a0;
                        }
                    }
                }
                __syncthreads();
            }
        if (tid < 32) {  // one warp compacts the sorted ids
            uint32_t nu = 0;
            for (uint32_t b0 = 0; b0 < na; b0 += 32) {
                const uint32_t i = b0 + lane;
                const bool keep = i < na && (i == 0 || acc[i] != acc[i - 1]);
                const uint32_t kb = __ballot_sync(0xFFFFFFFFu, keep);
                if (keep) resbuf[ro + nu + __popc(kb & ((1u << lane) - 1u))] = v.labels[acc[i]];
                nu += __popc(kb);
            }
            if (lane == 0) {
                res_count[qi] = nu;
                if (nu) atomicAdd(&ctr->n_result, (unsigned long long)nu);
            }
        }
    }
}

// Steps in flight per warp of the streaming kernel: 1 (64 registers, four blocks
// per SM) by default -- measured 13 % faster at 1M x 128 than 2 (two blocks per
// SM); HRNN_STREAM_STEPS=2 selects the other form.
int stream_steps() {
    static int s = 0;
    if (!s) {
        const char* e = std::getenv("HRNN_STREAM_STEPS");
        s = (e && e[0] == '2') ? 2 : 1;
    }
    return s;
}

template <class E, bool F, int NB, int S>
int chunks_per_sm() {
    static int per_sm = 0;
    if (!per_sm) {
        constexpr uint32_t dim = NB * 16;
        const size_t smem = 8 * verify_warp_smem(dim);
        auto k = k_verify_chunks<E, F, NB, S>;
        CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int ps = 1;
        CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ps, k, 256, smem));
        per_sm = std::max(ps, 1);
    }
    return per_sm;
}

template <class E, bool F, int NB, int S>
void launch_chunks(const DevView& v, const float* Q, uint32_t mmax, const uint32_t* prox, const uint32_t* plen,
                   const uint64_t* res_off, const float* kcol, uint32_t kidx, StreamBufs& B, uint64_t* resbuf,
                   SearchCounters* ctr, int nsm, cudaStream_t s) {
    constexpr uint32_t dim = NB * 16;
    const size_t smem = 8 * verify_warp_smem(dim);
    auto k = k_verify_chunks<E, F, NB, S>;
    k<<<(unsigned)(nsm * chunks_per_sm<E, F, NB, S>()), 256, smem, s>>>(
        v, Q, mmax, prox, plen, res_off, kcol, kidx, B.qq.as<int8_t>(), B.qmeta.as<float4>(), B.chunks.as<uint64_t>(),
        B.coff.as<uint64_t>() + B.npairs, B.ctl.as<uint32_t>(), B.acc_cnt.as<uint32_t>(), resbuf, ctr);
    CUDA_LAUNCH_CHECK();
}

}  // namespace

void stream_prepare(const DevView& v, bool wide, bool fused) {
    static bool big_set = false;
    if (!big_set) {
        CUDA_CHECK(cudaFuncSetAttribute(k_stream_finish_big, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)(kBigCap * 4)));
        big_set = true;
    }
    auto prep = [&](auto steps) {
        constexpr int S = decltype(steps)::value;
        if (v.dim == 128) {
            if (wide) fused ? chunks_per_sm<uint64_t, true, 8, S>() : chunks_per_sm<uint64_t, false, 8, S>();
            else fused ? chunks_per_sm<uint32_t, true, 8, S>() : chunks_per_sm<uint32_t, false, 8, S>();
        } else {
            if (wide) fused ? chunks_per_sm<uint64_t, true, 6, S>() : chunks_per_sm<uint64_t, false, 6, S>();
            else fused ? chunks_per_sm<uint32_t, true, 6, S>() : chunks_per_sm<uint32_t, false, 6, S>();
        }
    };
    if (stream_steps() == 1) prep(std::integral_constant<int, 1>{});
    else prep(std::integral_constant<int, 2>{});
}

bool stream_supported(const DevView& v) {
    return v.i8_screen && v.vec_i8 && v.lanes == 16 && (v.dim == 128 || v.dim == 96);
}

void StreamBufs::reserve(uint32_t nq_, uint32_t dim, size_t npairs_, size_t max_chunks) {
    qq.ensure((size_t)nq_ * dim + 16);
    qmeta.ensure((size_t)nq_ * 16 + 16);
    cnt.ensure((npairs_ + 1) * 4);
    coff.ensure((npairs_ + 1) * 8);
    chunks.ensure(std::max<size_t>(max_chunks, 1) * 8);
    acc_cnt.ensure((size_t)nq_ * 8 + 16);  // counts, then the list of queries for the block-wide pass
    ctl.ensure(64);
    npairs = npairs_;
}

size_t stream_max_chunks(uint64_t total_postings, size_t npairs) {
    return (size_t)(total_postings / kChunk) + npairs + 1;
}

void stream_verify(const DevView& v, bool wide, bool fused, const float* Q, uint32_t nq, uint32_t mmax,
                   const uint32_t* prox, const uint32_t* plen, const uint64_t* res_off, const float* kcol,
                   uint32_t kidx, uint64_t* resbuf, uint32_t* res_count, uint32_t* ovl, uint32_t* n_ovl,
                   SearchCounters* ctr, StreamBufs& B, int nsm, cudaStream_t s, const uint8_t* grp, uint8_t want) {
    const size_t npairs = (size_t)nq * mmax;
    if (B.npairs != npairs) fail(HRNN_ERR_STATE, "stream_verify: buffers reserved for another shape");
    stream_prepare(v, wide, fused);
    CUDA_CHECK(cudaMemsetAsync(B.acc_cnt.p, 0, (size_t)nq * 4, s));
    CUDA_CHECK(cudaMemsetAsync(B.ctl.p, 0, 16, s));
    k_meta_radius<<<(v.n + 255) / 256, 256, 0, s>>>(kcol, v.n, const_cast<float4*>(v.i8_meta));
    CUDA_LAUNCH_CHECK();
    k_quantize_queries<<<(unsigned)(((size_t)nq * 32 + 255) / 256), 256, 0, s>>>(Q, nq, v.dim, B.qq.as<int8_t>(),
                                                                                  B.qmeta.as<float4>());
    CUDA_LAUNCH_CHECK();
    k_chunk_count<<<(unsigned)((npairs + 255) / 256), 256, 0, s>>>(plen, npairs, B.cnt.as<uint32_t>());
    CUDA_LAUNCH_CHECK();
    CUDA_CHECK(cudaMemsetAsync(B.cnt.as<uint32_t>() + npairs, 0, 4, s));
    exclusive_scan_u32_to_u64(B.cnt.as<uint32_t>(), B.coff.as<uint64_t>(), npairs + 1, s, B.tmp);
    k_chunk_fill<<<(unsigned)((npairs + 255) / 256), 256, 0, s>>>(B.cnt.as<uint32_t>(), B.coff.as<uint64_t>(), npairs,
                                                                  B.chunks.as<uint64_t>());
    CUDA_LAUNCH_CHECK();
    auto go = [&](auto steps) {
        constexpr int S = decltype(steps)::value;
        auto run = [&](auto e, auto f, auto nb) {
            launch_chunks<decltype(e), decltype(f)::value, decltype(nb)::value, S>(v, Q, mmax, prox, plen, res_off,
                                                                                kcol, kidx, B, resbuf, ctr, nsm, s);
        };
        using T = std::true_type;
        using Fa = std::false_type;
        using N8 = std::integral_constant<int, 8>;
        using N6 = std::integral_constant<int, 6>;
        if (v.dim == 128) {
            if (wide) fused ? run(uint64_t{}, T{}, N8{}) : run(uint64_t{}, Fa{}, N8{});
            else fused ? run(uint32_t{}, T{}, N8{}) : run(uint32_t{}, Fa{}, N8{});
        } else {
            if (wide) fused ? run(uint64_t{}, T{}, N6{}) : run(uint64_t{}, Fa{}, N6{});
            else fused ? run(uint32_t{}, T{}, N6{}) : run(uint32_t{}, Fa{}, N6{});
        }
    };
    if (stream_steps() == 1) go(std::integral_constant<int, 1>{});
    else go(std::integral_constant<int, 2>{});
    uint32_t* big_n = B.ctl.as<uint32_t>() + 2;  // [2] big queries, [3] their work counter
    uint32_t* big = B.acc_cnt.as<uint32_t>() + nq;
    k_stream_finish<<<(nq + 7) / 8, 256, 0, s>>>(v, nq, res_off, B.acc_cnt.as<uint32_t>(), resbuf, res_count, big,
                                                 big_n, ctr, grp, want);
    CUDA_LAUNCH_CHECK();
    k_stream_finish_big<<<nsm, 1024, kBigCap * 4, s>>>(v, res_off, B.acc_cnt.as<uint32_t>(), big, big_n, big_n + 1,
                                                       resbuf, res_count, ovl, n_ovl, ctr);
    CUDA_LAUNCH_CHECK();
}

}  // namespace hrnn
