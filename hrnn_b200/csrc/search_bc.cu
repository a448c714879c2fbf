// Phase B + C of the batched search with one CTA per query (hrnn.h:2021-2070).
//
//   B: the reverse-list prefixes (rank < K') of the m proxies are scanned and the
//      owners deduplicated/counted in an open-address table in shared memory --
//      the reference's score_buf (hrnn.h:2029-2036).  To bound the table, the
//      owner-id space is cut into P ranges processed one after the other (every
//      posting is re-read P times; postings are 4 bytes, candidates 512).
//   C: every distinct owner whose count reaches the threshold (hrnn.h:2043-2052)
//      is verified in exact FP32, d(q,p) <= kdist(p, k-1) (hrnn.h:2058-2069):
//      the warps sweep the table, compact candidates with a ballot and verify four
//      per warp step (two per half-warp, loads issued together).  kdist(p, k-1) is
//      read from kcol, a per-call column of the KNN-slot radius (FLT_MAX when the
//      list is shorter than k, hrnn.h:290-291) that stays resident in L2.
//   Accepted ids of one range are sorted (bitonic, shared memory) and appended as
//   labels; ranges ascend, so the answer is in ascending internal-id order like
//   the reference's (hrnn.h:2055).
// A query whose table or accepted list overflows is flagged and answered by the
// global-memory warp kernel instead.
#include <cfloat>
#include <type_traits>

#include "beam.cuh"
#include "index.hpp"

namespace hrnn {

namespace {

// Candidate table: a power of two of slots, sized per query between 1024 and
// table_max for a load of at most 0.4 postings per slot; queries with more
// postings split the owner-id range into parts (one pass over the postings
// each, four postings per thread in flight).  Measured at m = 3 and 5, K' = 500:
// 4096 slots or 0.25 load take more passes and are slower; 16384 slots or 0.5 -
// 0.75 load take fewer passes but are slower too (more probes per insertion, and
// the larger shared-memory footprint leaves less L1 for the verified rows).
constexpr uint32_t kACap = 1024;      // accepted per range
constexpr int kBCThreads = 256;

template <class E>
__device__ __forceinline__ uint32_t owner_of(const void* ent, uint64_t i, uint32_t rb) {
    return (uint32_t)(((const E*)ent)[i] >> rb);
}

// Two exact distances per half-warp with the loads of both vectors in flight.
template <bool FUSED>
__device__ __forceinline__ void l2_half16_x2(const float* __restrict__ q, const float* __restrict__ x0,
                                             const float* __restrict__ x1, uint32_t nb, int l, float& d0,
                                             float& d1) {
    float a0 = 0.f, a1 = 0.f;
    uint32_t i = 0;
    for (; i + 4 <= nb; i += 4) {
        float u0 = __ldg(x0 + 16 * (i + 0) + l), u1 = __ldg(x0 + 16 * (i + 1) + l);
        float u2 = __ldg(x0 + 16 * (i + 2) + l), u3 = __ldg(x0 + 16 * (i + 3) + l);
        float w0 = __ldg(x1 + 16 * (i + 0) + l), w1 = __ldg(x1 + 16 * (i + 1) + l);
        float w2 = __ldg(x1 + 16 * (i + 2) + l), w3 = __ldg(x1 + 16 * (i + 3) + l);
        float q0 = q[16 * (i + 0) + l], q1 = q[16 * (i + 1) + l], q2 = q[16 * (i + 2) + l], q3 = q[16 * (i + 3) + l];
        a0 = sq_step(a0, q0 - u0, FUSED);
        a1 = sq_step(a1, q0 - w0, FUSED);
        a0 = sq_step(a0, q1 - u1, FUSED);
        a1 = sq_step(a1, q1 - w1, FUSED);
        a0 = sq_step(a0, q2 - u2, FUSED);
        a1 = sq_step(a1, q2 - w2, FUSED);
        a0 = sq_step(a0, q3 - u3, FUSED);
        a1 = sq_step(a1, q3 - w3, FUSED);
    }
    for (; i < nb; ++i) {
        float qq = q[16 * i + l];
        a0 = sq_step(a0, qq - __ldg(x0 + 16 * i + l), FUSED);
        a1 = sq_step(a1, qq - __ldg(x1 + 16 * i + l), FUSED);
    }
    float s0 = __shfl_sync(0xFFFFFFFFu, a0, 0, 16), s1 = __shfl_sync(0xFFFFFFFFu, a1, 0, 16);
#pragma unroll
    for (int k = 1; k < 16; ++k) {
        s0 = __fadd_rn(s0, __shfl_sync(0xFFFFFFFFu, a0, k, 16));
        s1 = __fadd_rn(s1, __shfl_sync(0xFFFFFFFFu, a1, k, 16));
    }
    d0 = s0;
    d1 = s1;
}

}  // namespace

__global__ void k_kdist_column(DevView v, uint32_t kidx, float* __restrict__ kcol) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= v.n) return;
    float kd;
    if (v.kdist_serve) {
        kd = v.kdist_serve[(size_t)i * v.mks + kidx];
    } else {
        uint32_t c = v.knn_hdr[i] & 0xFFFFu;
        kd = kidx >= c ? FLT_MAX : v.knn_dist[(size_t)i * v.K + kidx];
    }
    kcol[i] = kd;
}

__host__ __device__ constexpr uint32_t table_max(bool, bool) { return 8192; }

// dynamic shared memory: q[dim] | keys[H] | cnt[H] (threshold > 1 only) |
// stage[warps][32] | acc[kACap] | ctl[16] | q8 (dim bytes, padded to 16) | qm,
// H = table_max(counts, mixed)
__host__ size_t bc_cta_smem(uint32_t dim, bool counts, bool mixed) {
    const size_t H = table_max(counts, mixed);
    return (size_t)dim * 4 + H * 4 + (counts ? H * 4 : 0) + (kBCThreads / 32) * 64 * 4 + (size_t)kACap * 4 + 64 +
           (((size_t)dim + 15) & ~(size_t)15) + 16;
}

constexpr float kTieUlps = 16.f;  // FP64 re-decision band around the radius, in ulps of kd

template <class E, bool FUSED, bool COUNTS, bool MIXED>
__global__ void __launch_bounds__(kBCThreads) k_phase_bc_cta(
    DevView v, const float* __restrict__ Q, uint32_t nq, uint32_t mmax, const uint32_t* __restrict__ prox,
    const uint32_t* __restrict__ nprox, const uint32_t* __restrict__ plen, const uint64_t* __restrict__ qtotal,
    const uint64_t* __restrict__ res_off, float threshold, const float* __restrict__ kcol, uint32_t kidx,
    uint64_t* __restrict__ resbuf, uint32_t* __restrict__ res_count, uint32_t* __restrict__ next_q,
    uint32_t* __restrict__ overflow_list, uint32_t* __restrict__ n_overflow, SearchCounters* __restrict__ ctr) {
    extern __shared__ char smraw[];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    unsigned long long c_lowp = 0, c_fp32 = 0, c_fp64 = 0, c_flip = 0;
    constexpr int NW = kBCThreads / 32;
    float* q = (float*)smraw;
    uint32_t* keys = (uint32_t*)(q + v.dim);
    constexpr uint32_t HM = table_max(COUNTS, MIXED);
    uint32_t* cnt = keys + HM;
    uint32_t* stage = COUNTS ? cnt + HM : cnt;
    uint32_t* acc = stage + NW * 64;
    uint32_t* ctl = acc + kACap;  // 0: query, 1: accepted count, 2: overflow, 3: table full
    int* q8 = (int*)(ctl + 16);   // INT8 screen: the query as packed int8 words
    float4* qm = (float4*)((char*)q8 + ((v.dim + 15) & ~15u));  // (s_q^2 sum q8^2, s_q, ||q - s_q q8||, 0)
    const bool i8s = MIXED && v.i8_screen && v.vec_i8 != nullptr;
    unsigned long long c_post = 0, c_cand = 0, c_ver = 0, c_res = 0;
    const bool fast = v.lanes == 16 && (v.dim % 16) == 0;
    for (;;) {
        __syncthreads();
        if (tid == 0) ctl[0] = atomicAdd(next_q, 1u);
        __syncthreads();
        const uint32_t qi = ctl[0];
        if (qi >= nq) break;
        const uint64_t T = qtotal[qi];
        const uint32_t np_ = nprox[qi];
        if (T == 0) {
            if (tid == 0) res_count[qi] = 0;
            continue;
        }
        for (uint32_t i = tid; i < v.dim; i += kBCThreads) q[i] = Q[(size_t)qi * v.dim + i];
        if (i8s) {  // quantise the query for the INT8 screen (warp 0)
            __syncthreads();
            if (w == 0) {
                float mx = 0.f;
                for (uint32_t j = lane; j < v.dim; j += 32) mx = fmaxf(mx, fabsf(q[j]));
                for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
                const float sc = mx > 0.f ? mx / 127.f : 1.f;
                int8_t* qb = reinterpret_cast<int8_t*>(q8);
                double e2 = 0.0;
                int c2 = 0;
                for (uint32_t j = lane; j < v.dim; j += 32) {
                    const int c = max(-127, min(127, __float2int_rn(q[j] / sc)));
                    qb[j] = (int8_t)c;
                    const double dlt = (double)q[j] - (double)sc * (double)c;
                    e2 += dlt * dlt;
                    c2 += c * c;
                }
                for (int o = 16; o; o >>= 1) {
                    e2 += __shfl_xor_sync(0xFFFFFFFFu, e2, o);
                    c2 += __shfl_xor_sync(0xFFFFFFFFu, c2, o);
                }
                if (lane == 0) *qm = make_float4(sc * sc * (float)c2, sc, __double2float_ru(sqrt(e2)), 0.f);
            }
        }
        uint32_t HS = 1024;
        while (HS < HM && (uint64_t)HS * 2 / 5 < T) HS <<= 1;
        const uint32_t part_cap = HS * 2 / 5;
        const uint32_t P = (uint32_t)((T + part_cap - 1) / part_cap);
        const uint32_t width = (v.n + P - 1) / P;
        const uint64_t ro = res_off[qi];
        uint32_t written = 0;
        bool overflow = false;
        for (uint32_t part = 0; part < P && !overflow; ++part) {
            const uint32_t lo = part * width, hi = min(v.n, lo + width);
            for (uint32_t i = tid; i < HS; i += kBCThreads) {
                keys[i] = kInvalid;
                if (COUNTS) cnt[i] = 0;
            }
            if (tid == 0) {
                ctl[1] = 0;
                ctl[3] = 0;
            }
            __syncthreads();
            // ---- phase B: postings of this id range into the table ----
            for (uint32_t pi = 0; pi < np_; ++pi) {
                const uint32_t p = prox[(size_t)qi * mmax + pi];
                const uint32_t len = plen[(size_t)qi * mmax + pi];
                const uint64_t b = v.csr_off[p];
                if (part == 0) c_post += (tid == 0) ? len : 0;
                // four postings per thread loaded together, then inserted
                for (uint32_t e0 = tid; e0 < len; e0 += 4 * kBCThreads) {
                    uint32_t ow[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const uint32_t e = e0 + (uint32_t)u * kBCThreads;
                        ow[u] = e < len ? owner_of<E>(v.csr_ent, b + e, v.rank_bits) : hi;
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const uint32_t o = ow[u];
                        if (o < lo || o >= hi) continue;
                        uint32_t slot = hash32(o) & (HS - 1);
                        uint32_t probes = 0;
                        for (;;) {
                            uint32_t old = atomicCAS(&keys[slot], kInvalid, o);
                            if (old == kInvalid || old == o) {
                                if (COUNTS) atomicAdd(&cnt[slot], 1u);
                                break;
                            }
                            slot = (slot + 1) & (HS - 1);
                            if (++probes >= HS) {
                                ctl[3] = 1;
                                break;
                            }
                        }
                    }
                }
            }
            __syncthreads();
            if (ctl[3]) {
                overflow = true;
                break;
            }
            // ---- phase C: verify the table's candidates ----
            // Candidates are staged per warp until 32 are ready, then verified one
            // row per lane (32 rows in flight per warp).
            uint32_t* st = stage + w * 64;
            uint32_t ns = 0;
            auto accept = [&](uint32_t id) {
                const uint32_t pos = atomicAdd(&ctl[1], 1u);
                if (pos < kACap) acc[pos] = id;
            };
            // two lanes per row for the common dims (one memory round trip per 16
            // rows), one row per lane otherwise
            auto verify_pairs = [&](uint32_t cnt_, auto nbc) {
                constexpr int NB = decltype(nbc)::value;
                const int p = lane & 1;
                for (uint32_t r = 0; r < cnt_; r += 16) {
                    const uint32_t t = r + (lane >> 1);
                    const uint32_t id = st[t < cnt_ ? t : r];
                    const float kd = __ldg(kcol + id);
                    const float d = l2_pair16<FUSED, NB>(q, v.vec + (size_t)id * v.dim, p);
                    if (p == 0 && t < cnt_ && d <= kd) accept(id);
                }
            };
            // Mixed precision: a BF16 screen decides whatever its error bound allows;
            // the rest is decided in exact FP32 (the reference's order), and inside a
            // band of kTieUlps around the radius in FP64.
            auto verify_mixed = [&](uint32_t cnt_, auto nbc) {
                constexpr int NB = decltype(nbc)::value;
                const int p = lane & 1;
                for (uint32_t r = 0; r < cnt_; r += 16) {
                    const uint32_t t = r + (lane >> 1);
                    const bool live = t < cnt_;
                    const uint32_t id = st[live ? t : r];
                    const float kd = __ldg(kcol + id);
                    const float D = bf16_pair<NB>(q, v.vec_bf16 + (size_t)id * v.dim, p);
                    const float e = __ldg(v.vec_err + id);
                    // ||q - x|| is within e of ||q - bf16(x)|| (triangle inequality);
                    // rho covers the FP32 rounding of the screen's sum, of the
                    // reference's own sum and of this bound's few operations (each
                    // term is bounded by (dim + 8) * 2^-24 relative; 4x margin).
                    const float rho = (4.f * v.dim + 64.f) * 5.9604645e-8f;
                    const float sD = sqrtf(D);
                    const float hi = sD * (1.f + rho) + e, lo = fmaxf(0.f, sD * (1.f - rho) - e);
                    const float U = hi * hi * (1.f + rho), L = lo * lo * (1.f - rho);
                    int decision;  // 1 accept, 0 reject, -1 undecided (same in both lanes)
                    if (kd == FLT_MAX) decision = 1;
                    else if (U < kd) decision = 1;
                    else if (L > kd) decision = 0;
                    else decision = -1;
                    if (p == 0 && live && decision >= 0) c_lowp++;
                    const uint32_t und = __ballot_sync(0xFFFFFFFFu, live && decision < 0);
                    if (und) {  // exact FP32 for the undecided rows; all lanes take part
                        float d32 = l2_pair16<FUSED, NB>(q, v.vec + (size_t)id * v.dim, p);
                        d32 = __shfl_sync(0xFFFFFFFFu, d32, lane & ~1);
                        const bool tie = live && decision < 0 && v.knn_ids && kidx < (v.knn_hdr[id] & 0xFFFFu) &&
                                         fabsf(d32 - kd) <= kTieUlps * (nextafterf(kd, FLT_MAX) - kd);
                        if (live && decision < 0) {
                            decision = d32 <= kd;
                            if (p == 0) c_fp32++;
                        }
                        if (__any_sync(0xFFFFFFFFu, tie)) {
                            // FP64: d(q, x) against d(x, x_k), x_k the k-th neighbour of x
                            double a = 0.0, b = 0.0;
                            if (tie) {
                                const uint32_t nk = v.knn_ids[(size_t)id * v.K + kidx];
                                const float* x = v.vec + (size_t)id * v.dim;
                                const float* y = v.vec + (size_t)nk * v.dim;
                                for (uint32_t e2 = p; e2 < v.dim; e2 += 2) {
                                    const double tq = (double)q[e2] - (double)x[e2];
                                    const double ty = (double)x[e2] - (double)y[e2];
                                    a += tq * tq;
                                    b += ty * ty;
                                }
                            }
                            a += __shfl_xor_sync(0xFFFFFFFFu, a, 1);
                            b += __shfl_xor_sync(0xFFFFFFFFu, b, 1);
                            if (tie) {
                                const int d64 = a <= b;
                                if (p == 0) {
                                    c_fp64++;
                                    if (d64 != decision) c_flip++;
                                }
                                decision = d64;
                            }
                        }
                    }
                    if (p == 0 && live && decision == 1) accept(id);
                }
            };
            // INT8 screen (one row per lane, integer dot products) in front of the
            // BF16 one: |sqrt(d) - sqrt(D)| <= e_q + e_x with D = ||s_q q8 - s c||^2,
            // whose FP32 evaluation is within 8 ulps of (sqrt(s_q^2 sum q8^2) +
            // s sqrt(sum c^2))^2; what it cannot decide goes on to verify_mixed.
            auto verify_i8 = [&](uint32_t cnt_, auto nbc, auto nwc) {
                constexpr int NWW = decltype(nwc)::value;
                // Every lane loads a row below (the idle ones st[0]'s), so an empty
                // stage, whose st[0] was never written, loads nothing.  cnt_ is the
                // same in all lanes of the warp.
                if (cnt_ == 0) return;
                const bool live = (uint32_t)lane < cnt_;
                const uint32_t id = st[live ? lane : 0];
                const float kd = __ldg(kcol + id);
                const float4 xm = __ldg(v.i8_meta + id);
                const float4 qv = *qm;
                const float D = i8_row<NWW>(q8, qv, v.vec_i8 + (size_t)id * v.dim, xm);
                const float rq = sqrtf(qv.x), rx = xm.x * sqrtf(xm.z);
                const float ef = 8.f * 5.9604645e-8f * (rq + rx) * (rq + rx);
                const float e = qv.z + xm.y;
                const float rho = (4.f * v.dim + 64.f) * 5.9604645e-8f;
                const float hi = sqrtf(D + ef) * (1.f + rho) + e;
                const float lo = fmaxf(0.f, sqrtf(fmaxf(0.f, D - ef)) * (1.f - rho) - e);
                const float U = hi * hi * (1.f + rho), L = lo * lo * (1.f - rho);
                const int decision = kd == FLT_MAX ? 1 : (U < kd ? 1 : (L > kd ? 0 : -1));
                if (live && decision >= 0) c_lowp++;
                if (live && decision == 1) accept(id);
                const uint32_t und = __ballot_sync(0xFFFFFFFFu, live && decision < 0);
                __syncwarp();
                if (live && decision < 0) st[__popc(und & lanemask_lt())] = id;
                __syncwarp();
                if (und) verify_mixed((uint32_t)__popc(und), nbc);
            };
            auto verify = [&](uint32_t cnt_) {
                if (i8s && (v.dim == 128 || v.dim == 96)) {  // the dims with an unrolled BF16 screen behind it
                    if (v.dim == 128) verify_i8(cnt_, std::integral_constant<int, 8>{}, std::integral_constant<int, 8>{});
                    else verify_i8(cnt_, std::integral_constant<int, 6>{}, std::integral_constant<int, 6>{});
                    __syncwarp();
                    return;
                }
                if (MIXED && v.vec_bf16) {
                    if (v.dim == 128) verify_mixed(cnt_, std::integral_constant<int, 8>{});
                    else if (v.dim == 96) verify_mixed(cnt_, std::integral_constant<int, 6>{});
                    else if (v.dim == 256) verify_mixed(cnt_, std::integral_constant<int, 16>{});
                    else verify_pairs(cnt_, std::integral_constant<int, 8>{});  // unreachable: mixed needs 96/128/256
                    __syncwarp();
                    return;
                }
                if (fast && v.dim == 128) {
                    verify_pairs(cnt_, std::integral_constant<int, 8>{});
                } else if (fast && v.dim == 96) {
                    verify_pairs(cnt_, std::integral_constant<int, 6>{});
                } else if (fast && v.dim == 256) {
                    verify_pairs(cnt_, std::integral_constant<int, 16>{});
                } else if ((uint32_t)lane < cnt_) {
                    const uint32_t id = st[lane];
                    const float kd = __ldg(kcol + id);
                    const float* x = v.vec + (size_t)id * v.dim;
                    const float d = fast ? l2_row16<FUSED>(q, x, v.nb) : l2_thread(q, x, v.dim, v.lanes, v.fused);
                    if (d <= kd) accept(id);
                }
                __syncwarp();
            };
            for (uint32_t base = w * 32; base < HS; base += NW * 32) {
                const uint32_t s = base + lane;
                const uint32_t key = keys[s];
                bool valid = key != kInvalid;
                if (COUNTS && valid) valid = (float)cnt[s] >= threshold;
                const uint32_t nonempty = __ballot_sync(0xFFFFFFFFu, key != kInvalid);
                if (lane == 0) c_cand += __popc(nonempty);
                const uint32_t bal = __ballot_sync(0xFFFFFFFFu, valid);
                const uint32_t nv = __popc(bal);
                if (valid) st[ns + __popc(bal & lanemask_lt())] = key;
                __syncwarp();
                if (lane == 0) c_ver += nv;
                ns += nv;
                if (ns >= 32) {
                    verify(32);
                    const uint32_t rest = ns - 32;
                    const uint32_t mv = (uint32_t)lane < rest ? st[32 + lane] : 0;
                    __syncwarp();
                    if ((uint32_t)lane < rest) st[lane] = mv;
                    __syncwarp();
                    ns = rest;
                }
            }
            verify(ns);
            __syncthreads();
            const uint32_t na = ctl[1];
            if (na > kACap || ro + written + na > res_off[qi + 1]) {  // (or past a bounded slice)
                overflow = true;
                break;
            }
            // ---- sort this range's accepted ids, append labels ----
            uint32_t PP = 2;
            while (PP < na) PP <<= 1;
            for (uint32_t i = na + tid; i < PP; i += kBCThreads) acc[i] = kInvalid;
            __syncthreads();
            for (uint32_t k = 2; k <= PP; k <<= 1)
                for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                    for (uint32_t i = tid; i < PP; i += kBCThreads) {
                        uint32_t y = i ^ j;
                        if (y > i) {
                            uint32_t a = acc[i], c = acc[y];
                            if ((a > c) == ((i & k) == 0)) {
                                acc[i] = c;
                                acc[y] = a;
                            }
                        }
                    }
                    __syncthreads();
                }
            for (uint32_t i = tid; i < na; i += kBCThreads) resbuf[ro + written + i] = v.labels[acc[i]];
            written += na;
            __syncthreads();
        }
        if (tid == 0) {
            if (overflow) {
                overflow_list[atomicAdd(n_overflow, 1u)] = qi;
            } else {
                res_count[qi] = written;
                c_res += written;
            }
        }
    }
    if (lane == 0) {
        atomicAdd(&ctr->n_posting, c_post);
        atomicAdd(&ctr->n_cand, c_cand);
        atomicAdd(&ctr->n_verified, c_ver);
        atomicAdd(&ctr->n_result, c_res);
    }
    if (MIXED) {  // per-lane counts: reduce over the warp first
        for (int o = 16; o; o >>= 1) {
            c_lowp += __shfl_xor_sync(0xFFFFFFFFu, c_lowp, o);
            c_fp32 += __shfl_xor_sync(0xFFFFFFFFu, c_fp32, o);
            c_fp64 += __shfl_xor_sync(0xFFFFFFFFu, c_fp64, o);
            c_flip += __shfl_xor_sync(0xFFFFFFFFu, c_flip, o);
        }
        if (lane == 0) {
            atomicAdd(&ctr->n_lowp, c_lowp);
            atomicAdd(&ctr->n_fp32, c_fp32);
            atomicAdd(&ctr->n_fp64, c_fp64);
            atomicAdd(&ctr->n_flip, c_flip);
        }
    }
}

// explicit instantiations used by search_plain.cu
#define INST(E, F, C, X)                                                                                            \
    template __global__ void k_phase_bc_cta<E, F, C, X>(DevView, const float*, uint32_t, uint32_t, const uint32_t*, \
                                                        const uint32_t*, const uint32_t*, const uint64_t*,          \
                                                        const uint64_t*, float, const float*, uint32_t, uint64_t*,  \
                                                        uint32_t*, uint32_t*, uint32_t*, uint32_t*, SearchCounters*);
#define INST2(E, F, C) INST(E, F, C, false) INST(E, F, C, true)
INST2(uint32_t, false, false)
INST2(uint32_t, false, true)
INST2(uint32_t, true, false)
INST2(uint32_t, true, true)
INST2(uint64_t, false, false)
INST2(uint64_t, false, true)
INST2(uint64_t, true, false)
INST2(uint64_t, true, true)
#undef INST2
#undef INST

}  // namespace hrnn
