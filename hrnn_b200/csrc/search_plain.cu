// Batched RkNN search, plain form: answers bit-identical to the reference's
// searchRknn (hrnn.h:1966-2071) on the same index.
//
// Kernel A (one warp per query): greedy descent over the upper layers
// (hrnn.h:1992-2013) and the best-first base-layer search searchBaseLayerST
// (hrnn.h:484-616) with ef = max(ef_search, m), trimmed to the m nearest proxies
// (hrnn.h:2016-2019).  The beam formulation and its equivalence argument are in
// beam.cuh.
//
// Kernel B: length of each proxy's reverse-list prefix with rank < K' (binary
// search: segments are sorted by rank), and the per-query total.
//
// Kernel C (warp per query): phase B posting scan into a per-warp open-address
// table (the reference's score_buf counts), threshold filter and reset, exact
// FP32 verification against the stored kNN radius, results in ascending
// internal-id order (hrnn.h:2021-2070).
#include <algorithm>
#include <cstdlib>
#include <string>
#include <cfloat>
#include <vector>

#include "beam.cuh"
#include "beam_fast.cuh"
#include "index.hpp"
#include "mlp.hpp"
#include "plan.hpp"
#include "verify_stream.hpp"

namespace hrnn {

// search_bc.cu
template <class E, bool FUSED, bool COUNTS, bool MIXED>
__global__ void k_phase_bc_cta(DevView, const float*, uint32_t, uint32_t, const uint32_t*, const uint32_t*,
                               const uint32_t*, const uint64_t*, const uint64_t*, float, const float*, uint32_t,
                               uint64_t*, uint32_t*, uint32_t*, uint32_t*, uint32_t*, SearchCounters*);
using KCta = void (*)(DevView, const float*, uint32_t, uint32_t, const uint32_t*, const uint32_t*, const uint32_t*,
                      const uint64_t*, const uint64_t*, float, const float*, uint32_t, uint64_t*, uint32_t*,
                      uint32_t*, uint32_t*, uint32_t*, SearchCounters*);
template <class E>
KCta pick_bc(bool f, bool c, bool x) {
    if (x)
        return f ? (c ? k_phase_bc_cta<E, true, true, true> : k_phase_bc_cta<E, true, false, true>)
                 : (c ? k_phase_bc_cta<E, false, true, true> : k_phase_bc_cta<E, false, false, true>);
    return f ? (c ? k_phase_bc_cta<E, true, true, false> : k_phase_bc_cta<E, true, false, false>)
             : (c ? k_phase_bc_cta<E, false, true, false> : k_phase_bc_cta<E, false, false, false>);
}
void ensure_bf16(Index& ix);  // mixed.cu
void ensure_i8(Index& ix);    // mixed.cu
// budget.cu
__global__ void k_budget_features(DevView v, const float* Q, uint32_t nq, const uint32_t* prox, const float* proxd,
                                  const uint32_t* nprox, uint32_t stride, const float* kcol, const float* proj,
                                  float* feat);
__global__ void k_budget_decide(const float* z, uint32_t nq, float conf, uint32_t m0, uint32_t m1, const uint32_t* qm,
                                int rerun, uint32_t* nprox,
                                uint32_t* fb_list, uint32_t* fb_count, unsigned long long* levels, uint8_t* grp);
void ensure_projection(Index& ix, Budget& b);
__global__ void k_kdist_column(DevView v, uint32_t kidx, float* kcol);
size_t bc_cta_smem(uint32_t dim, bool counts, bool mixed);
// HRNN_VERIFY=table: the INT8 form verifies through the CTA table kernel as well
// (for comparisons of the two verification paths).
inline bool verify_table_forced() {
    const char* e = std::getenv("HRNN_VERIFY");
    return e && std::string(e) == "table";
}
// HRNN_LEARNED_SERIAL=1: the learned budget's second search and the verification
// run one after the other (for comparisons with the overlapped order).
inline bool learned_serial() {
    const char* e = std::getenv("HRNN_LEARNED_SERIAL");
    return e && e[0] == '1';
}

namespace {

// DM: distance mode of beam.cuh (0/1 exact FP32 unfused/fused, 2 BF16 rows, 3
// INT8 rows against the INT8-quantised query).
template <int DM>
__global__ void __launch_bounds__(128) k_phase_a(DevView v, const float* __restrict__ Q, uint32_t nq,
                                                 const uint32_t* __restrict__ qm, const uint32_t* __restrict__ qef,
                                                 uint32_t efc, uint32_t vc, uint32_t mmax,
                                                 uint32_t* __restrict__ prox, uint32_t* __restrict__ nprox,
                                                 SearchCounters* __restrict__ ctr,
                                                 const uint32_t* __restrict__ qlist, uint32_t m_over,
                                                 uint32_t ef_over, uint32_t m_keep, float* __restrict__ proxd,
                                                 uint32_t* __restrict__ next_q,
                                                 const uint32_t* __restrict__ nq_dev) {
    // qlist: search only the listed queries (nq = list length; nq_dev, when not
    // null, holds the length in device memory, at most nq -- a launch recorded
    // before the list is made); m_over / ef_over:
    // one (m, ef) for every query instead of the arrays (the beam is
    // max(ef, m) as in the reference); m_keep: write at least this many beam
    // entries (the learned budget's frontier; at most mmax); proxd: also write
    // the entries' distances.  next_q: work counter, zero at launch; a warp takes
    // the next query as soon as it finishes one.
    extern __shared__ char smem_raw[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    WarpSmem s = carve(smem_raw + (size_t)w * warp_smem_bytes(v.dim, efc, vc), v.dim, efc, vc);
    unsigned long long c_dist = 0, c_exp = 0;
    if (nq_dev) nq = min(nq, *nq_dev);
    for (;;) {
        uint32_t j = 0;
        if (lane == 0) j = atomicAdd(next_q, 1u);
        j = __shfl_sync(0xFFFFFFFFu, j, 0);
        if (j >= nq) break;
        const uint32_t qi = qlist ? qlist[j] : j;
        const uint32_t m = m_over ? m_over : qm[qi];
        const uint32_t EF = max(ef_over ? ef_over : qef[qi], m);
        if (v.n == 0 || m == 0) {
            if (lane == 0) nprox[qi] = 0;
            continue;
        }
        for (uint32_t i = lane; i < v.dim; i += 32) s.q[i] = Q[(size_t)qi * v.dim + i];
        __syncwarp();
        if constexpr (DM == 3) i8_prep_query(s, v.dim);
        uint32_t cur = v.enterpoint;
        float curd = warp_dist_one<DM>(v, s.q, cur);
        c_dist++;
        greedy_descent<DM>(v, s, v.maxlevel, 0, cur, curd, c_dist);
        c_dist++;  // the reference evaluates the entry point again (hrnn.h:505)
        uint32_t tsize = beam_search<DM>(v, s, cur, curd, EF, 0, vc, c_dist, c_exp);
        uint32_t np_ = min(min(max(m, m_keep), mmax), tsize);
        for (uint32_t i = lane; i < np_; i += 32) {
            prox[(size_t)qi * mmax + i] = s.ti[i] & kIdMask;
            if (proxd) proxd[(size_t)qi * mmax + i] = s.td[i];
        }
        if (lane == 0) nprox[qi] = np_;
        __syncwarp();
    }
    if (lane == 0) {
        atomicAdd(&ctr->n_dist, c_dist);
        atomicAdd(&ctr->n_expanded, c_exp);
    }
}

// Reduced-precision forms (DM 2 BF16, 3 INT8): descent, then the two-parent beam
// search of beam_fast.cuh.  Arguments as k_phase_a, plus:
//   save_cap, st_cnt / st_d / st_i: after the search, the first save_cap beam
//     entries (with their expanded flags) are stored per query (row stride
//     save_cap) -- the learned budget's frontier pass, which a fallback can
//     resume;
//   resume: start from the stored beam instead of the descent (its ids seed the
//     visited cache), continue with the query's own ef, store nothing;
//   nq_dev: as k_phase_a.
template <int DM, bool R2>
__global__ void __launch_bounds__(128, R2 ? 4 : 1) k_phase_a_fast(DevView v, const float* __restrict__ Q, uint32_t nq,
                                                      const uint32_t* __restrict__ qm,
                                                      const uint32_t* __restrict__ qef, uint32_t efc, uint32_t vc,
                                                      uint32_t mmax, uint32_t* __restrict__ prox,
                                                      uint32_t* __restrict__ nprox, SearchCounters* __restrict__ ctr,
                                                      const uint32_t* __restrict__ qlist, uint32_t m_over,
                                                      uint32_t ef_over, uint32_t m_keep, float* __restrict__ proxd,
                                                      uint32_t* __restrict__ next_q, uint32_t save_cap,
                                                      uint32_t* __restrict__ st_cnt, float* __restrict__ st_d,
                                                      uint32_t* __restrict__ st_i, int resume,
                                                      const uint32_t* __restrict__ nq_dev) {
    extern __shared__ char smem_raw[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    WarpSmem s = carve_fast(smem_raw + (size_t)w * fast_smem_bytes(v.dim, efc, vc), v.dim, efc, vc);
    unsigned long long c_dist = 0, c_exp = 0;
    if (nq_dev) nq = min(nq, *nq_dev);
    for (;;) {
        uint32_t j = 0;
        if (lane == 0) j = atomicAdd(next_q, 1u);
        j = __shfl_sync(0xFFFFFFFFu, j, 0);
        if (j >= nq) break;
        const uint32_t qi = qlist ? qlist[j] : j;
        const uint32_t m = m_over ? m_over : qm[qi];
        const uint32_t EF = min(max(ef_over ? ef_over : qef[qi], m), efc);
        if (v.n == 0 || m == 0) {
            if (lane == 0) nprox[qi] = 0;
            continue;
        }
        for (uint32_t i = lane; i < v.dim; i += 32) s.q[i] = Q[(size_t)qi * v.dim + i];
        for (uint32_t i = lane; i < vc; i += 32) s.vis[i] = kInvalid;
        __syncwarp();
        if constexpr (DM == 3) i8_prep_query(s, v.dim);
        uint32_t tsize;
        if (resume) {
            tsize = min(st_cnt[qi], EF);
            for (uint32_t i = lane; i < tsize; i += 32) {
                const uint32_t id = st_i[(size_t)qi * save_cap + i];
                s.td[i] = st_d[(size_t)qi * save_cap + i];
                s.ti[i] = id;
                s.vis[hash32(id & kIdMask) & (vc - 1)] = id & kIdMask;
            }
            __syncwarp();
        } else {
            uint32_t cur = v.enterpoint;
            float curd = warp_dist_one<DM>(v, s.q, cur);
            c_dist++;
            greedy_descent<DM>(v, s, v.maxlevel, 0, cur, curd, c_dist);
            if (lane == 0) {
                s.td[0] = curd;
                s.ti[0] = cur;
                s.vis[hash32(cur) & (vc - 1)] = cur;
            }
            __syncwarp();
            tsize = 1;
        }
        // a frontier pass that stores its beam keeps a reserve beyond EF for the
        // resumed search (expanding only the first EF entries)
        const uint32_t cap_beam = (save_cap && !resume) ? max(EF, min(save_cap, efc)) : EF;
        tsize = beam_search_fast<DM, R2>(v, s, tsize, cap_beam, EF, vc, c_dist, c_exp);
        if (save_cap && !resume) {
            const uint32_t ns = min(tsize, save_cap);
            for (uint32_t i = lane; i < ns; i += 32) {
                st_d[(size_t)qi * save_cap + i] = s.td[i];
                st_i[(size_t)qi * save_cap + i] = s.ti[i];
            }
            if (lane == 0) st_cnt[qi] = ns;
        }
        const uint32_t np_ = min(min(max(m, m_keep), mmax), tsize);
        for (uint32_t i = lane; i < np_; i += 32) {
            prox[(size_t)qi * mmax + i] = s.ti[i] & kIdMask;
            if (proxd) proxd[(size_t)qi * mmax + i] = s.td[i];
        }
        if (lane == 0) nprox[qi] = np_;
        __syncwarp();
    }
    if (lane == 0) {
        atomicAdd(&ctr->n_dist, c_dist);
        atomicAdd(&ctr->n_expanded, c_exp);
    }
}

template <class E>
__device__ __forceinline__ uint32_t entry_rank(const void* ent, uint64_t i, uint32_t rb) {
    return (uint32_t)(((const E*)ent)[i] & (E)((1ull << rb) - 1));
}
template <class E>
__device__ __forceinline__ uint32_t entry_owner(const void* ent, uint64_t i, uint32_t rb) {
    return (uint32_t)(((const E*)ent)[i] >> rb);
}

// Prefix length (rank < K') of every proxy's reverse list and the per-query total.
template <class E>
// grp (may be null): the queries with grp[q] != want get no postings (a batch
// verified in two groups).
__global__ void k_phase_b_count(DevView v, uint32_t nq, const uint32_t* __restrict__ Kp, uint32_t mmax,
                                const uint32_t* __restrict__ prox, const uint32_t* __restrict__ nprox,
                                uint32_t* __restrict__ plen, uint64_t* __restrict__ total,
                                const uint8_t* __restrict__ grp = nullptr, uint8_t want = 0) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t qi = (uint32_t)(t / mmax), pi = (uint32_t)(t % mmax);
    if (qi >= nq) return;
    uint32_t len = 0;
    if (pi < nprox[qi] && (!grp || grp[qi] == want)) {
        uint32_t p = prox[(size_t)qi * mmax + pi];
        uint64_t b = v.csr_off[p], e = v.csr_off[p + 1];
        uint32_t kp = Kp[qi];
        uint64_t lo = b, hi = e;  // first entry with rank >= K'
        while (lo < hi) {
            uint64_t mid = (lo + hi) >> 1;
            if (entry_rank<E>(v.csr_ent, mid, v.rank_bits) >= kp) hi = mid;
            else lo = mid + 1;
        }
        len = (uint32_t)(lo - b);
    }
    plen[t] = len;
    if (len) atomicAdd((unsigned long long*)&total[qi], (unsigned long long)len);
}

__device__ __forceinline__ float verify_kdist(const DevView& v, uint32_t id, uint32_t kidx) {
    if (v.kdist_serve) return v.kdist_serve[(size_t)id * v.mks + kidx];   // hrnn.h:287-288
    uint32_t cnt = v.knn_hdr[id] & 0xFFFFu;
    if (kidx >= cnt) return FLT_MAX;                                     // hrnn.h:290-291
    return v.knn_dist[(size_t)id * v.K + kidx];
}

// Phase B scan + phase C (hrnn.h:2021-2070), one warp per query.
template <class E, bool FUSED>
__global__ void __launch_bounds__(128) k_phase_bc(DevView v, const float* __restrict__ Q, uint32_t nq,
                                                  uint32_t mmax, const uint32_t* __restrict__ prox,
                                                  const uint32_t* __restrict__ nprox,
                                                  const uint32_t* __restrict__ plen,
                                                  const uint64_t* __restrict__ res_off, float threshold,
                                                  uint32_t kidx, uint32_t hcap, uint32_t* __restrict__ hkey_pool,
                                                  uint32_t* __restrict__ hcnt_pool, uint32_t* __restrict__ list_pool,
                                                  size_t list_stride, uint64_t* __restrict__ resbuf,
                                                  uint32_t* __restrict__ res_count, uint32_t* __restrict__ next_q,
                                                  const uint32_t* __restrict__ qlist,
                                                  SearchCounters* __restrict__ ctr,
                                                  const uint32_t* __restrict__ nq_dev,
                                                  uint32_t* __restrict__ clamp) {
    // nq_dev: the query count in device memory (a captured plan), else nq.
    // clamp (may be null): raised when a bounded result slice truncated an answer.
    extern __shared__ char smem_raw[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    const int half = lane >> 4, l = lane & 15;
    if (nq_dev) nq = *nq_dev;
    float* q = (float*)(smem_raw + (size_t)w * (v.dim * 4 + 16));
    uint32_t* nc_s = (uint32_t*)(q + v.dim);
    const size_t gw = (size_t)blockIdx.x * wpb + w;
    uint32_t* hkey = hkey_pool + gw * hcap;
    uint32_t* hcnt = hcnt_pool + gw * hcap;
    uint32_t* list = list_pool + gw * list_stride;
    unsigned long long c_post = 0, c_cand = 0, c_ver = 0, c_res = 0;
    for (;;) {
        uint32_t qi = 0;
        if (lane == 0) qi = atomicAdd(next_q, 1u);
        qi = __shfl_sync(0xFFFFFFFFu, qi, 0);
        if (qi >= nq) break;
        if (qlist) qi = qlist[qi];
        const uint32_t np_ = nprox[qi];
        for (uint32_t i = lane; i < v.dim; i += 32) q[i] = Q[(size_t)qi * v.dim + i];
        if (lane == 0) *nc_s = 0;
        __syncwarp();
        // Phase B: farthest proxy first, like the reference's heap pops.
        for (int pi = (int)np_ - 1; pi >= 0; --pi) {
            uint32_t p = prox[(size_t)qi * mmax + pi];
            uint32_t len = plen[(size_t)qi * mmax + pi];
            uint64_t b = v.csr_off[p];
            c_post += len;
            for (uint32_t e = lane; e < len; e += 32) {
                uint32_t owner = entry_owner<E>(v.csr_ent, b + e, v.rank_bits);
                uint32_t slot = hash32(owner) & (hcap - 1);
                for (;;) {
                    uint32_t old = atomicCAS(&hkey[slot], kInvalid, owner);
                    if (old == kInvalid) {
                        atomicAdd(&hcnt[slot], 1u);
                        list[atomicAdd(nc_s, 1u)] = slot;
                        break;
                    }
                    if (old == owner) {
                        atomicAdd(&hcnt[slot], 1u);
                        break;
                    }
                    slot = (slot + 1) & (hcap - 1);
                }
            }
        }
        __syncwarp();
        const uint32_t nc = *nc_s;
        c_cand += nc;
        // Phase C.1: threshold filter and table reset (hrnn.h:2043-2052).
        uint32_t nv = 0;
        for (uint32_t base = 0; base < nc; base += 32) {
            uint32_t i = base + lane;
            uint32_t id = kInvalid;
            bool keep = false;
            if (i < nc) {
                uint32_t slot = list[i];
                id = hkey[slot];
                keep = (float)hcnt[slot] >= threshold;
                hkey[slot] = kInvalid;
                hcnt[slot] = 0;
            }
            uint32_t kb = __ballot_sync(0xFFFFFFFFu, keep);
            __syncwarp();
            if (keep) list[nv + __popc(kb & lanemask_lt())] = id;
            nv += __popc(kb);
            __syncwarp();
        }
        c_ver += nv;
        // Phase C.2: exact FP32 verification (hrnn.h:2058-2069).
        uint32_t na = 0;
        if (v.lanes == 16 && v.dim % 16 == 0) {
            for (uint32_t r = 0; r < nv; r += 2) {
                uint32_t t = r + half;
                uint32_t id = list[t < nv ? t : r];
                float d = l2_half16<FUSED>(q, v.vec + (size_t)id * v.dim, v.nb, l);
                bool a = t < nv && d <= verify_kdist(v, id, kidx);
                uint32_t ab = __ballot_sync(0xFFFFFFFFu, a && l == 0);
                __syncwarp();
                if (lane == 0 && (ab & 1u)) list[na] = id;
                if (lane == 16 && (ab & (1u << 16))) list[na + (ab & 1u)] = id;
                na += __popc(ab);
                __syncwarp();
            }
        } else {
            for (uint32_t base = 0; base < nv; base += 32) {
                uint32_t i = base + lane;
                bool a = false;
                uint32_t id = 0;
                if (i < nv) {
                    id = list[i];
                    float d = l2_thread(q, v.vec + (size_t)id * v.dim, v.dim, v.lanes, v.fused);
                    a = d <= verify_kdist(v, id, kidx);
                }
                uint32_t ab = __ballot_sync(0xFFFFFFFFu, a);
                __syncwarp();
                if (a) list[na + __popc(ab & lanemask_lt())] = id;
                na += __popc(ab);
                __syncwarp();
            }
        }
        // Results in ascending internal-id order (hrnn.h:2055): rank sort.  A
        // bounded slice (a captured plan's staging) keeps its first entries and
        // raises *clamp.
        const uint64_t ro = res_off[qi];
        const uint64_t slice = res_off[qi + 1] - ro;
        const uint32_t room = (uint64_t)na < slice ? na : (uint32_t)slice;
        for (uint32_t i = lane; i < na; i += 32) {
            uint32_t x = list[i], rk = 0;
            for (uint32_t j = 0; j < na; ++j) rk += list[j] < x;
            if (rk < room) resbuf[ro + rk] = v.labels[x];
        }
        c_res += room;
        if (lane == 0) {
            res_count[qi] = room;
            if (room < na && clamp) atomicOr(clamp, 1u);
        }
        __syncwarp();
    }
    if (lane == 0) {
        atomicAdd(&ctr->n_posting, c_post);
        atomicAdd(&ctr->n_cand, c_cand);
        atomicAdd(&ctr->n_verified, c_ver);
        atomicAdd(&ctr->n_result, c_res);
    }
}

// grp (may be null): only the queries with grp[q] == want (a batch verified in two
// groups, each with its own staging).
__global__ void k_pack_results(uint32_t nq, const uint64_t* __restrict__ res_off,
                               const uint32_t* __restrict__ res_count, const uint64_t* __restrict__ out_off,
                               const uint64_t* __restrict__ resbuf, uint64_t* __restrict__ out,
                               const uint8_t* __restrict__ grp = nullptr, uint8_t want = 0) {
    uint32_t qi = blockIdx.x;
    if (qi >= nq || (grp && grp[qi] != want)) return;
    uint32_t c = res_count[qi];
    for (uint32_t i = threadIdx.x; i < c; i += blockDim.x) out[out_off[qi] + i] = resbuf[res_off[qi] + i];
}

__global__ void k_l2_pairs(const float* a, const float* b, size_t n, uint32_t dim, int lanes, int fused,
                           float* out) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = l2_thread(a + i * dim, b + i * dim, dim, lanes, fused);
}

int sms(int dev) {
    int v = 148;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v;
}

// Captured plans: each query's m and ef clamped to the plan's maxima (flag set
// when one was above), so the beam and the proxy table never outgrow their sizes.
__global__ void k_plan_inputs(const uint32_t* __restrict__ m_in, const uint32_t* __restrict__ ef_in, uint32_t nq,
                              uint32_t m_max, uint32_t ef_max, uint32_t* __restrict__ m_out,
                              uint32_t* __restrict__ ef_out, uint32_t* __restrict__ flag) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nq) return;
    const uint32_t m = m_in[i], ef = ef_in[i];
    if (m > m_max || ef > ef_max) atomicOr(flag, 1u);
    m_out[i] = min(m, m_max);
    ef_out[i] = min(ef, ef_max);
}

// k_pack_results when the total (out_off[nq]) fits the caller's capacity.
__global__ void k_pack_results_capped(uint32_t nq, const uint64_t* __restrict__ res_off,
                                      const uint32_t* __restrict__ res_count, const uint64_t* __restrict__ out_off,
                                      const uint64_t* __restrict__ resbuf, uint64_t* __restrict__ out, size_t cap) {
    const uint32_t qi = blockIdx.x;
    if (qi >= nq || out_off[nq] > cap) return;
    const uint32_t c = res_count[qi];
    for (uint32_t i = threadIdx.x; i < c; i += blockDim.x) out[out_off[qi] + i] = resbuf[res_off[qi] + i];
}

}  // namespace

DevView make_view(Index& ix) {
    DevView v{};
    v.vec = ix.vec.as<float>();
    v.adj0 = ix.adj0.as<uint32_t>();
    v.upper = ix.d_upper.as<uint32_t>();
    v.upper_off = ix.d_upper_off.as<uint64_t>();
    v.knn_hdr = ix.knn_hdr.as<uint32_t>();
    v.knn_dist = ix.knn_dist.as<float>();
    v.kdist_serve = ix.serve_mode ? ix.kdist_serve.as<float>() : nullptr;
    v.csr_off = ix.csr_off.as<uint64_t>();
    v.csr_ent = ix.csr_ent.p;
    v.labels = ix.labels.as<uint64_t>();
    v.vec_bf16 = ix.bf16_valid ? ix.vec_bf16.as<uint16_t>() : nullptr;
    v.vec_err = ix.bf16_valid ? ix.vec_norm.as<float>() : nullptr;
    v.vec_i8 = ix.i8_valid ? ix.vec_i8.as<int8_t>() : nullptr;
    v.i8_meta = ix.i8_valid ? ix.i8_meta.as<float4>() : nullptr;
    v.knn_ids = ix.knn_ids.as<uint32_t>();
    v.n = (uint32_t)ix.cur;
    v.dim = (uint32_t)ix.dim;
    v.nb = (uint32_t)(ix.dim / 16);
    v.W0 = (uint32_t)(1 + ix.maxM0);
    v.WU = (uint32_t)(1 + ix.maxM);
    v.K = (uint32_t)ix.K;
    v.mks = (uint32_t)ix.max_k_serve;
    v.rank_bits = ix.rank_bits;
    v.maxlevel = ix.maxlevel;
    v.enterpoint = ix.enterpoint;
    v.wide = ix.wide;
    v.lanes = ix.order.lanes;
    v.fused = ix.order.fused;
    return v;
}

// The phase-A kernel of a batch: distance mode dm (0/1 exact FP32, 2 BF16, 3
// INT8), the reference-order beam (k_phase_a) or, for the reduced-precision
// forms, the two-parent search (k_phase_a_fast; r2: its INT8 two-rows-per-lane
// shape); the batch's queries, parameter arrays and proxy outputs.
struct PhaseA {
    bool fast;
    int dm;
    bool r2;
    DevView v;
    const float* q;
    const uint32_t *qm, *qef;
    uint32_t efc, mmax;
    uint32_t *prox, *nprox;
    SearchCounters* ctr;
};

static const void* phase_a_kernel(bool fast, int dm, bool r2) {
    return fast ? (dm == 3 ? (r2 ? (const void*)k_phase_a_fast<3, true> : (const void*)k_phase_a_fast<3, false>)
                           : (const void*)k_phase_a_fast<2, false>)
                : (dm == 3 ? (const void*)k_phase_a<3>
                           : dm == 2 ? (const void*)k_phase_a<2>
                                     : dm == 1 ? (const void*)k_phase_a<1> : (const void*)k_phase_a<0>);
}

// One launch; qlist / m_over / ef_over / m_keep / proxd / save / resume / nq_dev as
// documented at k_phase_a_fast (the exact kernel takes no save or resume).
static void launch_phase_a(const PhaseA& p, unsigned g, int cw, uint32_t cv, size_t sm, cudaStream_t ls, uint32_t nqq,
                    const uint32_t* qlist, uint32_t m_over, uint32_t ef_over, uint32_t m_keep, float* proxd,
                    uint32_t* ctrq, uint32_t save_cap, uint32_t* st_cnt, float* st_d, uint32_t* st_i, int resume,
                    const uint32_t* nq_dev) {
    if (p.fast) {
        auto k = p.dm == 3 ? (p.r2 ? k_phase_a_fast<3, true> : k_phase_a_fast<3, false>) : k_phase_a_fast<2, false>;
        k<<<g, cw * 32, sm, ls>>>(p.v, p.q, nqq, p.qm, p.qef, p.efc, cv, p.mmax, p.prox, p.nprox, p.ctr, qlist, m_over,
                                  ef_over, m_keep, proxd, ctrq, save_cap, st_cnt, st_d, st_i, resume, nq_dev);
    } else {
        auto k = p.dm == 3 ? k_phase_a<3> : p.dm == 2 ? k_phase_a<2> : p.dm == 1 ? k_phase_a<1> : k_phase_a<0>;
        k<<<g, cw * 32, sm, ls>>>(p.v, p.q, nqq, p.qm, p.qef, p.efc, cv, p.mmax, p.prox, p.nprox, p.ctr, qlist, m_over,
                                  ef_over, m_keep, proxd, ctrq, nq_dev);
    }
    CUDA_LAUNCH_CHECK();
}

uint64_t search_batch(Index& ix, const SearchArgs& a) {
    if (!ix.rknng_built) fail(HRNN_ERR_STATE, "searchRknn: RKNNG not built");
    ensure_flat_rknng(ix);
    cudaStream_t s = a.stream ? a.stream : ix.stream;
    const size_t nq = a.nq;
    if (ix.serve_mode && (a.k == 0 || a.k > ix.max_k_serve))
        fail(HRNN_ERR_ARG, "searchRknn: k must be in [1, max_k_serve] in serve mode");
    ix.sync_upper_to_device();
    cudaEvent_t ev[4];
    for (auto& e : ev) CUDA_CHECK(cudaEventCreate(&e));
    CUDA_CHECK(cudaMemsetAsync(ix.counters.p, 0, sizeof(SearchCounters), s));
    const unsigned long long launches0 = launch_counter().load();
    if (nq == 0) {
        CUDA_CHECK(cudaMemsetAsync(a.d_out_offsets, 0, 8, s));
        CUDA_CHECK(cudaStreamSynchronize(s));
        for (auto& e : ev) cudaEventDestroy(e);
        ix.last_stats = hrnn_search_stats{};
        return 0;
    }
    // Per-batch maxima of m and ef (sizes the proxy table and the beam).
    uint32_t mmax = 1, efmax = 1;
    if (a.h_mmax) {
        mmax = std::max<uint32_t>(1, a.h_mmax);
        efmax = std::max<uint32_t>(1, std::max(a.h_efmax, a.h_mmax));
    } else {
        std::vector<uint32_t> hm(nq), hef(nq);
        CUDA_CHECK(cudaMemcpyAsync(hm.data(), a.d_m, nq * 4, cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaMemcpyAsync(hef.data(), a.d_ef, nq * 4, cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaStreamSynchronize(s));
        for (size_t i = 0; i < nq; ++i) {
            mmax = std::max(mmax, hm[i]);
            efmax = std::max(efmax, std::max(hef[i], hm[i]));
        }
    }
    if (efmax > (1u << 16)) fail(HRNN_ERR_ARG, "searchRknn: ef_search/m too large (max 65536)");
    const bool learned = ix.budget && ix.budget->enabled && ix.budget->mlp.ready && ix.dim % 4 == 0;
    // Learned budget: the frontier keeps kFrontier beam entries; with a level ef
    // (two-pass mode) the frontier beam is that ef.
    const bool two_pass = learned && ix.budget->ef > 0;
    if (learned) mmax = std::max<uint32_t>(mmax, kFrontier);
    // two-pass mode: the frontier pass stores its beam with a reserve beyond the
    // level ef for the second search to resume (the reduced-precision forms); the
    // batch's beam capacity holds it, so the stored beam does not depend on the
    // batch's largest ef
    const uint32_t reserve = two_pass ? (std::max(2 * ix.budget->ef, ix.budget->ef + 32) + 31) & ~31u : 0;
    if (two_pass) efmax = std::max<uint32_t>(efmax, reserve);
    DevView v = make_view(ix);
    const uint32_t efc = (efmax + 31) & ~31u;
    // Visited-cache slots (lossy; a miss costs a recomputed row).  1024 rather than
    // more: the smaller per-warp shared memory keeps more warps resident, which
    // pays for the ~10% extra rows at ef = 200.
    uint32_t vc = 512;
    size_t wsm = std::max(warp_smem_bytes(v.dim, efc, vc), fast_smem_bytes(v.dim, efc, vc));
    int wpb = (int)std::max<size_t>(1, std::min<size_t>(4, (200 * 1024) / wsm));
    size_t smem_a = wsm * wpb;
    DevMem& prox = ix.scratch[0];
    DevMem& nprox = ix.scratch[1];
    DevMem& plen = ix.scratch[2];
    DevMem& qtot = ix.scratch[3];
    DevMem& tmp = ix.scratch[4];
    prox.ensure(nq * mmax * 4);
    nprox.ensure(nq * 4);
    plen.ensure(nq * mmax * 4);
    qtot.ensure((nq + 1) * 8 * 4 + (nq + 1) * 4 * 2 + 128);  // d_total2 / d_resoff2 after d_next
    uint64_t* d_total = qtot.as<uint64_t>();
    uint64_t* d_resoff = d_total + (nq + 1);
    uint32_t* d_rcount = (uint32_t*)(d_resoff + (nq + 1));
    uint32_t* d_next = d_rcount + (nq + 1);
    CUDA_CHECK(cudaMemsetAsync(d_total, 0, (nq + 1) * 8, s));
    CUDA_CHECK(cudaMemsetAsync(d_rcount, 0, (nq + 1) * 4 + 32, s));  // and the 8 counters after it
    SearchCounters* ctr = ix.counters.as<SearchCounters>();
    const bool fusedsimd = (ix.order.fused & 1) != 0;
    // Mixed precision (hrnn_set_precision): BF16 rows for the beam and the
    // verification screen; decisions still exact (FP32 / FP64 band).
    const bool mixed = (ix.precision == HRNN_PREC_BF16 || ix.precision == HRNN_PREC_INT8) &&
                       (v.dim == 96 || v.dim == 128 || v.dim == 256) && v.lanes == 16;
    const bool int8 = ix.precision == HRNN_PREC_INT8 && v.dim % 16 == 0 && v.dim <= 256;
    if (mixed) ensure_bf16(ix);
    if (int8) ensure_i8(ix);
    if (mixed || int8) v = make_view(ix);
    v.i8_screen = (mixed && int8) ? 1 : 0;
    const int nsm = sms(ix.device);
    // Learned budget, two-pass, INT8 streaming verification: the second search (the
    // queries the MLP is not confident about) runs on a second stream beside the
    // verification of the other queries, which verify as group 0; the second
    // search's queries verify afterwards as group 1.  grp[q] is the query's group.
    const bool counts_mode = a.threshold > 1.0f;
    const bool stream_bc = int8 && mixed && !counts_mode && stream_supported(v) && !verify_table_forced();
    bool split = false;
    uint8_t* grp = nullptr;
    CUDA_CHECK(cudaEventRecord(ev[0], s));
    {
        // The exact form runs the reference-order beam (k_phase_a); the reduced-
        // precision forms the two-parent search (k_phase_a_fast).
        // (The two-parent search reads link rows of at most 33 words, maxM0 <= 32.)
        const bool fast = (int8 || mixed) && v.W0 <= 33;
        const int dm = int8 ? 3 : mixed ? 2 : fusedsimd ? 1 : 0;
        // r2: the INT8 two-parent search loads all 64 rows of a step at once (a launch-shape choice)
        bool r2 = false;
        auto kfun_of = [&](bool two) { return phase_a_kernel(fast, dm, two); };
        auto smem_for = [&](uint32_t cv, int cw) {
            return (fast ? fast_smem_bytes(v.dim, efc, cv) : warp_smem_bytes(v.dim, efc, cv)) * (size_t)cw;
        };
        // One launch of the form's phase-A kernel; qlist / ef_over / m_keep / proxd /
        // save / resume as documented at k_phase_a_fast (the exact kernel takes no
        // save or resume).
        cudaStream_t ls = s;  // the stream of `launch` (the second search may run beside the first group's verification)
        auto launch = [&](unsigned g, int cw, uint32_t cv, size_t sm, uint32_t nqq, const uint32_t* qlist,
                          uint32_t m_over, uint32_t ef_over, uint32_t m_keep, float* proxd, uint32_t* ctrq,
                          uint32_t save_cap, uint32_t* st_cnt, float* st_d, uint32_t* st_i, int resume) {
            PhaseA pa{fast, dm, r2, v, a.d_q, a.d_m, a.d_ef, efc, mmax, prox.as<uint32_t>(), nprox.as<uint32_t>(), ctr};
            launch_phase_a(pa, g, cw, cv, sm, ls, nqq, qlist, m_over, ef_over, m_keep, proxd, ctrq, save_cap, st_cnt,
                           st_d, st_i, resume, nullptr);
        };
        uint32_t* d_qa = d_next + 4;  // work counters of the phase-A launches (zeroed with d_rcount)
        // Launch shape: the tuned one of this (distance mode, beam size), else timed
        // now on this batch when autotuning is on and the batch is large enough.
        const uint64_t shape_key = ((uint64_t)dm << 32) | efc;
        auto shape = ix.autotune ? ix.a_shape.find(shape_key) : ix.a_shape.end();
        if (shape != ix.a_shape.end()) {
            wpb = (int)(shape->second.first & 0xFF);
            r2 = (shape->second.first & 0x100) != 0;
            vc = shape->second.second;
        } else if (ix.autotune && !learned && nq >= 1024) {
            float best = FLT_MAX;
            int bw = wpb;
            uint32_t bv = vc;
            bool br2 = false;
            cudaEvent_t t0, t1;
            CUDA_CHECK(cudaEventCreate(&t0));
            CUDA_CHECK(cudaEventCreate(&t1));
            for (int two = 0; two < ((fast && dm == 3) ? 2 : 1); ++two)
            for (uint32_t cv : {256u, 512u, 1024u}) {
                for (int cw : {2, 4}) {
                    const size_t sm = smem_for(cv, cw);
                    if (sm > 200 * 1024) continue;
                    r2 = two != 0;
                    const void* kfun = kfun_of(r2);
                    CUDA_CHECK(cudaFuncSetAttribute(kfun, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
                    int ps = 1;
                    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ps, kfun, cw * 32, sm));
                    const unsigned g = (unsigned)std::max<size_t>(
                        1, std::min<size_t>((nq + cw - 1) / cw, (size_t)nsm * std::max(ps, 1)));
                    CUDA_CHECK(cudaMemsetAsync(d_qa, 0, 4, s));
                    CUDA_CHECK(cudaEventRecord(t0, s));
                    launch(g, cw, cv, sm, (uint32_t)nq, nullptr, 0, 0, 0, nullptr, d_qa, 0, nullptr, nullptr,
                           nullptr, 0);
                    CUDA_CHECK(cudaEventRecord(t1, s));
                    CUDA_CHECK(cudaEventSynchronize(t1));
                    float ms = 0.f;
                    CUDA_CHECK(cudaEventElapsedTime(&ms, t0, t1));
                    if (ms < best) {
                        best = ms;
                        bw = cw;
                        bv = cv;
                        br2 = r2;
                    }
                }
            }
            cudaEventDestroy(t0);
            cudaEventDestroy(t1);
            wpb = bw;
            vc = bv;
            r2 = br2;
            ix.a_shape[shape_key] = {(uint32_t)wpb | (r2 ? 0x100u : 0u), vc};
            // the trials' counts and work counter start over
            CUDA_CHECK(cudaMemsetAsync(ctr, 0, sizeof(SearchCounters), s));
            CUDA_CHECK(cudaMemsetAsync(d_qa, 0, 4, s));
            CUDA_CHECK(cudaEventRecord(ev[0], s));
        }
        smem_a = smem_for(vc, wpb);
        if (smem_a > 227 * 1024) fail(HRNN_ERR_ARG, "searchRknn: ef/dim too large for one warp's beam");
        const void* kfun = kfun_of(r2);
        CUDA_CHECK(cudaFuncSetAttribute(kfun, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_a));
        // Persistent grid (every resident block), queries handed out by counters.
        int per_sm = 1;
        CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfun, wpb * 32, smem_a));
        auto grid_for = [&](size_t n) {
            return (unsigned)std::max<size_t>(1, std::min<size_t>((n + wpb - 1) / wpb, (size_t)nsm * std::max(per_sm, 1)));
        };
        if (!learned) {
            launch(grid_for(nq), wpb, vc, smem_a, (uint32_t)nq, nullptr, 0, 0, 0, nullptr, d_qa, 0, nullptr, nullptr,
                   nullptr, 0);
        } else {
            // Learned budget: frontier pass for every query, features, MLP,
            // decision.  Single-pass mode: the frontier is the caller's own beam,
            // levels only trim the proxies.  Two-pass mode: the frontier beam is
            // the level ef; the queries the MLP is not confident about continue
            // that search with the caller's (m, ef) -- the two-parent search
            // resumes from the stored beam (the exact form searches again).
            Budget& b = *ix.budget;
            ensure_projection(ix, b);
            ix.kcol.ensure((size_t)std::max<size_t>(ix.cur, 1) * 4);
            k_kdist_column<<<(unsigned)((ix.cur + 255) / 256), 256, 0, s>>>(v, (uint32_t)(a.k - 1), ix.kcol.as<float>());
            CUDA_LAUNCH_CHECK();
            b.feat.ensure(nq * kMlpIn * 4);
            b.proxd.ensure(nq * mmax * 4);
            b.fallback_list.ensure(nq * 4 + 64);
            b.decided.ensure(64);
            uint32_t* fb_count = b.decided.as<uint32_t>();
            unsigned long long* levels = (unsigned long long*)(b.decided.as<char>() + 8);
            CUDA_CHECK(cudaMemsetAsync(b.decided.p, 0, 64, s));
            // the stored frontier beam: the level beam plus a reserve (twice the
            // level ef, at least 32 more entries) that the fallback resumes
            const uint32_t save_cap = (two_pass && fast) ? reserve : 0;
            uint32_t *st_cnt = nullptr, *st_i = nullptr;
            float* st_d = nullptr;
            if (save_cap) {
                b.saved.ensure(nq * 4 + (size_t)nq * save_cap * 8 + 256);
                st_cnt = b.saved.as<uint32_t>();
                st_d = (float*)(b.saved.as<char>() + ((nq * 4 + 255) & ~(size_t)255));
                st_i = (uint32_t*)(st_d + (size_t)nq * save_cap);
            }
            launch(grid_for(nq), wpb, vc, smem_a, (uint32_t)nq, nullptr, two_pass ? b.m[1] : 0, two_pass ? b.ef : 0,
                   kFrontier, b.proxd.as<float>(), d_qa, save_cap, st_cnt, st_d, st_i, 0);
            k_budget_features<<<(unsigned)((nq * 32 + 255) / 256), 256, 0, s>>>(
                v, a.d_q, (uint32_t)nq, prox.as<uint32_t>(), b.proxd.as<float>(), nprox.as<uint32_t>(), mmax,
                ix.kcol.as<float>(), b.proj.as<float>(), b.feat.as<float>());
            CUDA_LAUNCH_CHECK();
            b.mlp.forward(b.feat.as<float>(), (int)nq, s);
            const bool may_split = two_pass && fast && stream_bc && !learned_serial();
            if (may_split) {
                ix.scratch[9].ensure(nq + 16);
                grp = ix.scratch[9].as<uint8_t>();
            }
            k_budget_decide<<<(unsigned)((nq + 255) / 256), 256, 0, s>>>(
                b.mlp.z3.as<float>(), (uint32_t)nq, b.confidence, b.m[0], b.m[1], a.d_m, two_pass ? 1 : 0,
                nprox.as<uint32_t>(), b.fallback_list.as<uint32_t>(), fb_count, levels, grp);
            CUDA_LAUNCH_CHECK();
            if (two_pass) {
                uint32_t nfb = 0;
                CUDA_CHECK(cudaMemcpyAsync(&nfb, fb_count, 4, cudaMemcpyDeviceToHost, s));
                CUDA_CHECK(cudaStreamSynchronize(s));
                split = may_split && nfb > 0 && nfb < nq;
                if (split) {
                    if (!ix.aux) CUDA_CHECK(cudaStreamCreateWithFlags(&ix.aux, cudaStreamNonBlocking));
                    for (auto& e : ix.aux_ev)
                        if (!e) CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
                    CUDA_CHECK(cudaEventRecord(ix.aux_ev[0], s));
                    CUDA_CHECK(cudaStreamWaitEvent(ix.aux, ix.aux_ev[0], 0));
                    ls = ix.aux;
                }
                if (nfb)
                    launch(grid_for(nfb), wpb, vc, smem_a, nfb, b.fallback_list.as<uint32_t>(), 0, 0, 0, nullptr,
                           d_qa + 1, save_cap, st_cnt, st_d, st_i, save_cap ? 1 : 0);
                if (split) {
                    CUDA_CHECK(cudaEventRecord(ix.aux_ev[1], ix.aux));
                    ls = s;
                }
            }
        }
    }
    CUDA_CHECK(cudaEventRecord(ev[1], s));
    // Phase B (posting counts, staging) and C (verification) of the queries with
    // g[q] == want (all of them for g null), staged in `resm` at offsets d_off.
    auto run_bc = [&](const uint8_t* g, uint8_t want, uint64_t* d_tot, uint64_t* d_off, DevMem& resm,
                      bool first) -> uint64_t* {
        {
            size_t tot = nq * mmax;
            auto kern = ix.wide ? k_phase_b_count<uint64_t> : k_phase_b_count<uint32_t>;
            kern<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(v, (uint32_t)nq, a.d_Kp, mmax, prox.as<uint32_t>(),
                                                               nprox.as<uint32_t>(), plen.as<uint32_t>(), d_tot, g,
                                                               want);
            CUDA_LAUNCH_CHECK();
        }
        exclusive_scan_u64(d_tot, d_off, nq + 1, s, tmp);
        std::vector<uint64_t> htot(nq);
        uint64_t sum_total = 0;
        CUDA_CHECK(cudaMemcpyAsync(htot.data(), d_tot, nq * 8, cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaMemcpyAsync(&sum_total, d_off + nq, 8, cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaStreamSynchronize(s));
        DevMem& hkey = ix.scratch[5];
        DevMem& hcnt = ix.scratch[6];
        const size_t res_bytes = std::max<uint64_t>(sum_total, 1) * 8;
        resm.ensure(res_bytes + (nq + 1) * 4 + 256);
        uint64_t* rbuf = resm.as<uint64_t>();
        uint32_t* ovl = (uint32_t*)(resm.as<char>() + ((res_bytes + 255) & ~(size_t)255));
        uint32_t* d_nov = d_next + 1;  // spare counters after d_next, zeroed with d_rcount
        if (first) CUDA_CHECK(cudaEventRecord(ev[2], s));
        // Per-call column of kdist(p, k-1) (hrnn.h:286-293), then the verification.
        const uint32_t kidx = (uint32_t)(a.k - 1);
        if (first) {
            ix.kcol.ensure((size_t)std::max<size_t>(ix.cur, 1) * 4);
            k_kdist_column<<<(unsigned)((ix.cur + 255) / 256), 256, 0, s>>>(v, kidx, ix.kcol.as<float>());
            CUDA_LAUNCH_CHECK();
        }
        if (stream_bc) {
            // INT8 form: postings verified as they are read, in chunks spread over
            // persistent warps
            const size_t npairs = nq * mmax;
            ix.sb.reserve((uint32_t)nq, v.dim, npairs, stream_max_chunks(sum_total, npairs));
            stream_verify(v, ix.wide, fusedsimd, a.d_q, (uint32_t)nq, mmax, prox.as<uint32_t>(), plen.as<uint32_t>(),
                          d_off, ix.kcol.as<float>(), kidx, rbuf, d_rcount, ovl, d_nov, ctr, ix.sb, nsm, s, g, want);
        } else {
            // one CTA per query (every query: the CTA path verifies a batch in one group)
            const size_t smem = bc_cta_smem(v.dim, counts_mode, mixed);
            KCta kc = ix.wide ? pick_bc<uint64_t>(fusedsimd, counts_mode, mixed)
                              : pick_bc<uint32_t>(fusedsimd, counts_mode, mixed);
            CUDA_CHECK(cudaFuncSetAttribute(kc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            int per_sm = 1;
            CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kc, 256, smem));
            unsigned grid = (unsigned)std::min<size_t>(nq, (size_t)nsm * std::max(per_sm, 1));
            kc<<<grid, 256, smem, s>>>(v, a.d_q, (uint32_t)nq, mmax, prox.as<uint32_t>(), nprox.as<uint32_t>(),
                                       plen.as<uint32_t>(), d_tot, d_off, a.threshold, ix.kcol.as<float>(), kidx,
                                       rbuf, d_rcount, d_next, ovl, d_nov, ctr);
            CUDA_LAUNCH_CHECK();
        }
        // Queries whose shared-memory table or accepted list overflowed: the
        // global-memory warp kernel, with a table sized for their posting count.
        uint32_t nov = 0;
        CUDA_CHECK(cudaMemcpyAsync(&nov, d_nov, 4, cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaStreamSynchronize(s));
        if (nov) {
            std::vector<uint32_t> hov(nov);
            CUDA_CHECK(cudaMemcpy(hov.data(), ovl, nov * 4, cudaMemcpyDeviceToHost));
            uint64_t tmax = 1;
            for (uint32_t qi : hov) tmax = std::max(tmax, htot[qi]);
            uint32_t hcap = 64;
            while (hcap < 2 * tmax) hcap <<= 1;
            size_t per_slot = (size_t)hcap * 8 + tmax * 4;
            size_t slots = std::max<size_t>(1, std::min<size_t>((size_t)nsm * 8 * 4, (size_t)(4ull << 30) / per_slot));
            slots = std::min<size_t>(slots, ((size_t)nov + 3) / 4 * 4);
            slots = (slots + 3) / 4 * 4;
            size_t need_h = slots * (size_t)hcap * 4;
            if (hkey.bytes < need_h) {
                hkey.alloc(need_h);
                hcnt.alloc(need_h);
                CUDA_CHECK(cudaMemsetAsync(hkey.p, 0xFF, need_h, s));
                CUDA_CHECK(cudaMemsetAsync(hcnt.p, 0, need_h, s));
            }
            DevMem& lp = ix.scratch[4];
            lp.ensure(slots * tmax * 4 + 64);
            uint32_t* d_next2 = d_next + 2;
            CUDA_CHECK(cudaMemsetAsync(d_next2, 0, 4, s));
            size_t smem_w = 4 * (v.dim * 4 + 16);
            void (*kern)(DevView, const float*, uint32_t, uint32_t, const uint32_t*, const uint32_t*, const uint32_t*,
                         const uint64_t*, float, uint32_t, uint32_t, uint32_t*, uint32_t*, uint32_t*, size_t,
                         uint64_t*, uint32_t*, uint32_t*, const uint32_t*, SearchCounters*, const uint32_t*,
                         uint32_t*);
            if (ix.wide) kern = fusedsimd ? k_phase_bc<uint64_t, true> : k_phase_bc<uint64_t, false>;
            else kern = fusedsimd ? k_phase_bc<uint32_t, true> : k_phase_bc<uint32_t, false>;
            kern<<<(unsigned)(slots / 4), 128, smem_w, s>>>(v, a.d_q, nov, mmax, prox.as<uint32_t>(),
                                                            nprox.as<uint32_t>(), plen.as<uint32_t>(), d_off,
                                                            a.threshold, kidx, hcap, hkey.as<uint32_t>(),
                                                            hcnt.as<uint32_t>(), lp.as<uint32_t>(), (size_t)tmax,
                                                            rbuf, d_rcount, d_next2, ovl, ctr, nullptr, nullptr);
            CUDA_LAUNCH_CHECK();
        }
        return rbuf;
    };
    uint64_t* resbuf = run_bc(split ? grp : nullptr, 0, d_total, d_resoff, ix.scratch[7], true);
    uint64_t *resbuf2 = nullptr, *d_total2 = nullptr, *d_resoff2 = nullptr;
    if (split) {
        // group 1 once its second search is done
        // after d_next's max(nq + 1, 8) counters, 8-byte aligned
        const uintptr_t at = (uintptr_t)(d_next + std::max<size_t>(nq + 1, 8));
        d_total2 = (uint64_t*)((at + 7) & ~(uintptr_t)7);
        d_resoff2 = d_total2 + (nq + 1);
        CUDA_CHECK(cudaStreamWaitEvent(s, ix.aux_ev[1], 0));
        CUDA_CHECK(cudaMemsetAsync(d_total2, 0, (nq + 1) * 8, s));
        CUDA_CHECK(cudaMemsetAsync(d_next, 0, 12, s));  // the verification's counters of group 0
        resbuf2 = run_bc(grp, 1, d_total2, d_resoff2, ix.scratch[8], false);
    }
    exclusive_scan_u32_to_u64(d_rcount, a.d_out_offsets, nq + 1, s, tmp);
    uint64_t total = 0;
    CUDA_CHECK(cudaMemcpyAsync(&total, a.d_out_offsets + nq, 8, cudaMemcpyDeviceToHost, s));
    CUDA_CHECK(cudaStreamSynchronize(s));
    if (total <= a.cap && total > 0) {
        k_pack_results<<<(unsigned)nq, 128, 0, s>>>((uint32_t)nq, d_resoff, d_rcount, a.d_out_offsets, resbuf,
                                                     a.d_out_labels, split ? grp : nullptr, 0);
        CUDA_LAUNCH_CHECK();
        if (split) {
            k_pack_results<<<(unsigned)nq, 128, 0, s>>>((uint32_t)nq, d_resoff2, d_rcount, a.d_out_offsets, resbuf2,
                                                         a.d_out_labels, grp, 1);
            CUDA_LAUNCH_CHECK();
        }
    }
    CUDA_CHECK(cudaEventRecord(ev[3], s));
    CUDA_CHECK(cudaStreamSynchronize(s));
    SearchCounters hc{};
    CUDA_CHECK(cudaMemcpy(&hc, ix.counters.p, sizeof(hc), cudaMemcpyDeviceToHost));
    if (learned) {
        CUDA_CHECK(cudaMemcpy(ix.budget->n_level, ix.budget->decided.as<char>() + 8, 24, cudaMemcpyDeviceToHost));
        ix.budget->mlp.check_tc();
    }
    hrnn_search_stats st{};
    st.n_queries = nq;
    st.n_dist = hc.n_dist;
    st.n_expanded = hc.n_expanded;
    st.n_posting = hc.n_posting;
    st.n_cand = hc.n_cand;
    st.n_verified = hc.n_verified;
    st.n_result = hc.n_result;
    st.n_lowp_decided = hc.n_lowp;
    st.n_fp32_decided = hc.n_fp32;
    st.n_fp64_decided = hc.n_fp64;
    st.n_fp64_flipped = hc.n_flip;
    st.n_launches = launch_counter().load() - launches0;
    if (learned)
        for (int i = 0; i < 3; ++i) st.n_budget[i] = ix.budget->n_level[i];
    float t01 = 0, t12 = 0, t23 = 0;
    cudaEventElapsedTime(&t01, ev[0], ev[1]);
    cudaEventElapsedTime(&t12, ev[1], ev[2]);
    cudaEventElapsedTime(&t23, ev[2], ev[3]);
    st.a_warps_per_block = (uint32_t)wpb;
    st.a_visit_slots = vc;
    st.phase_a_ms = t01;
    st.phase_b_ms = t12;
    st.phase_c_ms = t23;
    ix.last_stats = st;
    for (auto& e : ev) cudaEventDestroy(e);
    return total;
}

void l2_batch_device(const float* a, const float* b, size_t n, size_t dim, L2Order o, float* out,
                     cudaStream_t s) {
    if (!n) return;
    k_l2_pairs<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(a, b, n, (uint32_t)dim, o.lanes, o.fused, out);
    CUDA_LAUNCH_CHECK();
}

void kdist_column(Index& ix, uint32_t k, float* host_out) {
    if (!ix.knng_built && !ix.serve_mode) fail(HRNN_ERR_STATE, "kdist: KNNG not built yet");
    if (k == 0 || (ix.serve_mode ? k > ix.max_k_serve : k > ix.K)) fail(HRNN_ERR_ARG, "kdist: k out of range");
    if (ix.cur == 0) return;
    DevView v = make_view(ix);
    cudaStream_t s = ix.stream;
    ix.kcol.ensure(ix.cur * 4);
    k_kdist_column<<<(unsigned)((ix.cur + 255) / 256), 256, 0, s>>>(v, k - 1, ix.kcol.as<float>());
    CUDA_LAUNCH_CHECK();
    CUDA_CHECK(cudaMemcpyAsync(host_out, ix.kcol.p, ix.cur * 4, cudaMemcpyDeviceToHost, s));
    CUDA_CHECK(cudaStreamSynchronize(s));
}

Budget& budget_of(Index& ix) {
    if (!ix.budget) ix.budget.reset(new Budget());
    return *ix.budget;
}

// Features of nq queries (device buffers) as the learned search computes them:
// the frontier pass of a search with (m, ef) -- (m1, level ef) in two-pass mode --
// and k_budget_features, in the index's precision mode.
void budget_features(Index& ix, const float* d_q, size_t nq, uint32_t k, uint32_t m, uint32_t ef, float* d_feat) {
    if (!ix.rknng_built) fail(HRNN_ERR_STATE, "searchRknn: RKNNG not built");
    ensure_flat_rknng(ix);
    if (ix.dim % 4 != 0) fail(HRNN_ERR_ARG, "budget: dim must be a multiple of 4");
    if (nq == 0) return;
    Budget& b = budget_of(ix);
    if (b.ef > 0) {
        m = b.m[1];
        ef = b.ef;
    }
    if (m == 0 || std::max(m, ef) > (1u << 16)) fail(HRNN_ERR_ARG, "budget_features: need 1 <= m, ef <= 65536");
    cudaStream_t s = ix.stream;
    ix.sync_upper_to_device();
    const bool mixed = (ix.precision == HRNN_PREC_BF16 || ix.precision == HRNN_PREC_INT8) &&
                       (ix.dim == 96 || ix.dim == 128 || ix.dim == 256) && ix.order.lanes == 16;
    const bool int8 = ix.precision == HRNN_PREC_INT8 && ix.dim % 16 == 0 && ix.dim <= 256;
    if (mixed) ensure_bf16(ix);
    if (int8) ensure_i8(ix);
    DevView v = make_view(ix);
    ensure_projection(ix, b);
    const uint32_t mmax = std::max<uint32_t>(m, kFrontier), efc = (std::max(m, ef) + 31) & ~31u, vc = 1024;
    const bool fast = (mixed || int8) && v.W0 <= 33;  // the search the learned form's frontier pass runs
    const size_t wsm = fast ? fast_smem_bytes(v.dim, efc, vc) : warp_smem_bytes(v.dim, efc, vc);
    const int wpb = (int)std::max<size_t>(1, std::min<size_t>(4, (200 * 1024) / wsm));
    const size_t smem_a = wsm * wpb;
    if (smem_a > 227 * 1024) fail(HRNN_ERR_ARG, "budget: ef/dim too large for one warp's beam");
    DevMem prox, nprox, proxd, next;
    prox.alloc(nq * mmax * 4);
    nprox.alloc(nq * 4);
    proxd.alloc(nq * mmax * 4);
    next.alloc(16);
    CUDA_CHECK(cudaMemsetAsync(next.p, 0, 16, s));
    ix.kcol.ensure((size_t)std::max<size_t>(ix.cur, 1) * 4);
    k_kdist_column<<<(unsigned)((ix.cur + 255) / 256), 256, 0, s>>>(v, k - 1, ix.kcol.as<float>());
    CUDA_LAUNCH_CHECK();
    const int nsm = sms(ix.device);
    unsigned grid = (unsigned)std::max<size_t>(1, std::min<size_t>((nq + wpb - 1) / wpb, (size_t)nsm * 16));
    if (fast) {
        auto kern = int8 ? k_phase_a_fast<3, false> : k_phase_a_fast<2, false>;
        CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_a));
        kern<<<grid, wpb * 32, smem_a, s>>>(v, d_q, (uint32_t)nq, nullptr, nullptr, efc, vc, mmax,
                                            prox.as<uint32_t>(), nprox.as<uint32_t>(),
                                            ix.counters.as<SearchCounters>(), nullptr, m, ef, kFrontier,
                                            proxd.as<float>(), next.as<uint32_t>(), 0, nullptr, nullptr, nullptr, 0,
                                            nullptr);
    } else {
        auto kern = int8 ? k_phase_a<3> : mixed ? k_phase_a<2> : ((ix.order.fused & 1) != 0) ? k_phase_a<1> : k_phase_a<0>;
        CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_a));
        kern<<<grid, wpb * 32, smem_a, s>>>(v, d_q, (uint32_t)nq, nullptr, nullptr, efc, vc, mmax,
                                            prox.as<uint32_t>(), nprox.as<uint32_t>(),
                                            ix.counters.as<SearchCounters>(), nullptr, m, ef, kFrontier,
                                            proxd.as<float>(), next.as<uint32_t>(), nullptr);
    }
    CUDA_LAUNCH_CHECK();
    k_budget_features<<<(unsigned)((nq * 32 + 255) / 256), 256, 0, s>>>(v, d_q, (uint32_t)nq, prox.as<uint32_t>(),
                                                                       proxd.as<float>(), nprox.as<uint32_t>(), mmax,
                                                                       ix.kcol.as<float>(), b.proj.as<float>(), d_feat);
    CUDA_LAUNCH_CHECK();
    CUDA_CHECK(cudaStreamSynchronize(s));
}

// ---- captured search plans ---------------------------------------------------
//
// The sequence of search_batch for one batch shape, with its four host reads
// replaced by bounds fixed at creation:
//   - the maxima of m and ef: the plan's m_max / ef_max (inputs clamped on the
//     device, k_plan_inputs);
//   - the result staging size: nq * m_max * (longest reverse list), an upper bound
//     of every query's posting count;
//   - the overflow count: the overflow kernel always runs, reads the count from
//     device memory and sizes its tables for the same bound;
//   - the total before packing: k_pack_results_capped checks it on the device.
// Device layout of qtot as in search_batch: total[nq+1] u64 | res_off[nq+1] u64 |
// rcount[nq+1] u32 | counters u32[8] (BC work, overflow count, overflow work,
// -, phase-A work x2, -, -).

namespace {

// mmax: the bound of a query's verified proxies (m_max); mstride: the row stride
// of the proxy arrays (the learned budget's frontier keeps kFrontier entries).
struct PlanLaunch {
    uint32_t efc, vc, mmax, mstride, reserve, wpb, grid_a, grid_bc, kidx, slots, hcap;
    size_t smem_a, smem_bc, smem_w, tmax;
    bool mixed, int8, fusedsimd, counts, fast, r2, learned, two_pass;
};

PlanLaunch plan_launch_shape(Index& ix, const SearchPlan& p) {
    PlanLaunch L{};
    DevView v = make_view(ix);
    L.mmax = std::max<uint32_t>(1, p.m_max);
    // the learned budget as search_batch runs it: frontier pass, MLP, and in
    // two-pass mode (level ef > 0) a second search of the other queries
    L.learned = ix.budget && ix.budget->enabled && ix.budget->mlp.ready && ix.dim % 4 == 0;
    L.two_pass = L.learned && ix.budget->ef > 0;
    L.mstride = L.learned ? std::max<uint32_t>(L.mmax, kFrontier) : L.mmax;
    uint32_t efmax = std::max(std::max<uint32_t>(1, p.ef_max), L.mmax);
    L.reserve = L.two_pass ? (std::max(2 * ix.budget->ef, ix.budget->ef + 32) + 31) & ~31u : 0;  // as search_batch
    if (L.two_pass) efmax = std::max(efmax, L.reserve);
    L.efc = (efmax + 31) & ~31u;
    L.vc = 512;
    L.fusedsimd = (ix.order.fused & 1) != 0;
    L.mixed = (ix.precision == HRNN_PREC_BF16 || ix.precision == HRNN_PREC_INT8) &&
              (v.dim == 96 || v.dim == 128 || v.dim == 256) && v.lanes == 16;
    L.int8 = ix.precision == HRNN_PREC_INT8 && v.dim % 16 == 0 && v.dim <= 256;
    L.fast = (L.mixed || L.int8) && v.W0 <= 33;  // the reduced-precision forms' two-parent search, as in search_batch
    auto wsm_of = [&](uint32_t vc) {
        return L.fast ? fast_smem_bytes(v.dim, L.efc, vc) : warp_smem_bytes(v.dim, L.efc, vc);
    };
    L.wpb = (uint32_t)std::max<size_t>(1, std::min<size_t>(4, (200 * 1024) / wsm_of(L.vc)));
    L.smem_a = wsm_of(L.vc) * L.wpb;
    const uint64_t shape_key = ((uint64_t)(L.int8 ? 3 : L.mixed ? 2 : L.fusedsimd ? 1 : 0) << 32) | L.efc;
    auto shape = ix.autotune ? ix.a_shape.find(shape_key) : ix.a_shape.end();  // tuned by an earlier batch call
    if (shape != ix.a_shape.end()) {
        L.wpb = shape->second.first & 0xFF;
        L.r2 = (shape->second.first & 0x100) != 0;
        L.vc = shape->second.second;
        L.smem_a = wsm_of(L.vc) * L.wpb;
    }
    L.counts = p.threshold > 1.0f;
    L.kidx = p.k - 1;
    L.smem_bc = bc_cta_smem(v.dim, L.counts, L.mixed);
    L.smem_w = 4 * (v.dim * 4 + 16);
    return L;
}

}  // namespace

// The smallest result slice of a captured plan (>= the finishing passes' 16384).
constexpr size_t kPlanMinSlice = 16384;

// Slice lengths of a captured plan: each query's posting count, at most qcap.
__global__ void k_cap_totals(const uint64_t* __restrict__ total, uint32_t n, uint64_t qcap, uint64_t* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = min(total[i], qcap);
}

// A plan verified in two groups: group 1's slices follow group 0's (*base: group
// 0's total, its offsets' last entry).
__global__ void k_add_base(uint64_t* __restrict__ off, uint32_t n, const uint64_t* __restrict__ base) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) off[i] += *base;
}

// Each query's slice offset from its group's offsets.
__global__ void k_merge_offsets(const uint8_t* __restrict__ grp, uint32_t nq, const uint64_t* __restrict__ off0,
                                const uint64_t* __restrict__ off1, uint64_t* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nq) out[i] = grp[i] ? off1[i] : off0[i];
}

void plan_create(SearchPlan& p, cudaStream_t s) {
    Index& ix = *p.ix;
    if (!ix.rknng_built) fail(HRNN_ERR_STATE, "searchRknn: RKNNG not built");
    ensure_flat_rknng(ix);
    if (p.nq == 0 || p.nq > (1u << 30)) fail(HRNN_ERR_ARG, "search plan: nq must be in [1, 2^30]");
    if (p.m_max == 0 || p.ef_max == 0) fail(HRNN_ERR_ARG, "search plan: m_max and ef_max must be >= 1");
    if (std::max(p.m_max, p.ef_max) > (1u << 16)) fail(HRNN_ERR_ARG, "searchRknn: ef_search/m too large (max 65536)");
    if (p.k == 0) fail(HRNN_ERR_ARG, "search plan: k must be >= 1");
    if (ix.serve_mode && p.k > ix.max_k_serve) fail(HRNN_ERR_ARG, "searchRknn: k must be in [1, max_k_serve] in serve mode");
    ix.sync_upper_to_device();
    PlanLaunch L = plan_launch_shape(ix, p);
    if (L.smem_a > 227 * 1024) fail(HRNN_ERR_ARG, "searchRknn: ef/dim too large for one warp's beam");
    if (L.mixed) ensure_bf16(ix);
    if (L.int8) ensure_i8(ix);
    DevView v = make_view(ix);
    v.i8_screen = (L.mixed && L.int8) ? 1 : 0;
    const size_t nq = p.nq;
    // longest reverse list: bounds every proxy's posting prefix
    std::vector<uint64_t> off(ix.cur + 1);
    CUDA_CHECK(cudaMemcpy(off.data(), ix.csr_off.p, off.size() * 8, cudaMemcpyDeviceToHost));
    uint64_t maxdeg = 1;
    for (size_t i = 0; i < ix.cur; ++i) maxdeg = std::max<uint64_t>(maxdeg, off[i + 1] - off[i]);
    L.tmax = (size_t)L.mmax * maxdeg;
    // Result staging: every query's slice holds its postings, up to qcap -- the
    // full bound nq * m_max * (longest reverse list) where it takes at most a
    // quarter of the free memory, else as many as fit (at least kPlanMinSlice).  A
    // query whose acceptances pass its slice is answered by the overflow pass; an
    // answer longer than its slice is cut and raises the clamp flag.
    size_t free_b = 0, total_b = 0;
    CUDA_CHECK(cudaMemGetInfo(&free_b, &total_b));
    size_t qcap = L.tmax;
    if (nq * qcap * 8 > free_b / 4) qcap = std::max<size_t>(kPlanMinSlice, (free_b / 4) / (nq * 8));
    qcap = std::min(qcap, L.tmax);
    if (const char* e = std::getenv("HRNN_PLAN_MAX_SLICE")) {  // a smaller bound (tests of the bounded path)
        const size_t v = std::strtoull(e, nullptr, 10);
        if (v >= 1) qcap = std::min(qcap, v);
    }
    const size_t res_entries = nq * qcap;
    if (res_entries * 8 > free_b / 2)
        fail(HRNN_ERR_NOMEM, "search plan: the result staging (nq * 16384 entries at least) does not fit; lower nq");
    const int nsm = sms(ix.device);
    // overflow tables: a fixed pool of warp slots, each sized for the bound
    uint32_t hcap = 64;
    while (hcap < 2 * L.tmax) hcap <<= 1;
    L.hcap = hcap;
    const size_t per_slot = (size_t)hcap * 8 + L.tmax * 4;
    size_t slots = std::max<size_t>(4, std::min<size_t>((size_t)nsm * 4, (free_b / 8) / per_slot) / 4 * 4);
    L.slots = (uint32_t)slots;
    // verification: the streaming kernel of the INT8 form where search_batch takes it, else the CTA kernel
    const bool stream = L.int8 && L.mixed && !L.counts && stream_supported(v) && !verify_table_forced();
    // learned budget, two-pass, streaming verification: the second search runs on
    // a second stream beside the verification of the confident queries (group 0),
    // and its queries verify afterwards as group 1 (as search_batch)
    const bool split = L.two_pass && L.fast && stream && !learned_serial();
    // buffers
    p.inputs.alloc((3 * nq + 8) * 4);  // m | ef | flag, 3 spare | overflow list
    p.prox.alloc(nq * L.mstride * 4);
    p.nprox.alloc(nq * 4);
    p.plen.alloc(nq * L.mstride * 4);
    p.qtot.alloc((nq + 1) * 8 * 3 + (nq + 1) * 4 + 64);
    p.res.alloc(std::max<size_t>(res_entries, 1) * 8);
    p.kcol.alloc(std::max<size_t>(ix.cur, 1) * 4);
    p.hkey.alloc(slots * hcap * 4);
    p.hcnt.alloc(slots * hcap * 4);
    p.lp.alloc(slots * L.tmax * 4 + 64);
    p.ctr.alloc(sizeof(SearchCounters));
    CUDA_CHECK(cudaMemsetAsync(p.hkey.p, 0xFF, p.hkey.bytes, s));
    CUDA_CHECK(cudaMemsetAsync(p.hcnt.p, 0, p.hcnt.bytes, s));
    CUDA_CHECK(cudaMemsetAsync(p.qtot.p, 0, p.qtot.bytes, s));
    uint64_t* d_total = p.qtot.as<uint64_t>();
    uint64_t* d_resoff = d_total + (nq + 1);
    uint32_t* d_rcount = (uint32_t*)(d_resoff + (nq + 1));
    uint32_t* d_next = d_rcount + (nq + 1);
    uint64_t* d_totc = (uint64_t*)(d_next + 8 + ((nq + 1) & 1));  // per-query slice lengths (8-byte aligned)
    uint32_t* pm = p.inputs.as<uint32_t>();
    uint32_t* pef = pm + nq;
    uint32_t* flag = pef + nq;
    // learned budget: features, MLP activations, frontier distances, decisions,
    // stored frontier beams, groups and group 1's totals / offsets
    Budget* bud = L.learned ? ix.budget.get() : nullptr;
    uint32_t save_cap = 0;
    uint32_t *fb_list = nullptr, *fb_count = nullptr, *st_cnt = nullptr, *st_i = nullptr;
    float *feat = nullptr, *proxd = nullptr, *st_d = nullptr, *mlpw = nullptr;
    unsigned long long* levels = nullptr;
    uint8_t* grp = nullptr;
    uint64_t *d_total2 = nullptr, *d_totc2 = nullptr, *d_resoff2 = nullptr, *d_resoffm = nullptr;
    if (bud) {
        ensure_projection(ix, *bud);
        save_cap = (L.two_pass && L.fast) ? L.reserve : 0;
        p.lfeat.alloc(nq * kMlpIn * 4);
        p.lmlp.alloc(nq * (kMlpIn + 4 * kMlpH + kMlpOut) * 4);
        p.lproxd.alloc(nq * L.mstride * 4);
        p.lfb.alloc(nq * 4 + 64);
        p.lgrp.alloc(nq + 16);
        p.loff.alloc((nq + 1) * 8 * 4);
        if (save_cap) p.lsaved.alloc(nq * 4 + (size_t)nq * save_cap * 8 + 256);
        feat = p.lfeat.as<float>();
        mlpw = p.lmlp.as<float>();
        proxd = p.lproxd.as<float>();
        fb_count = p.lfb.as<uint32_t>();                                  // [0] count, [2..7] level counts
        levels = (unsigned long long*)(p.lfb.as<char>() + 8);
        fb_list = p.lfb.as<uint32_t>() + 16;
        grp = split ? p.lgrp.as<uint8_t>() : nullptr;
        d_total2 = p.loff.as<uint64_t>();
        d_totc2 = d_total2 + (nq + 1);
        d_resoff2 = d_totc2 + (nq + 1);
        d_resoffm = d_resoff2 + (nq + 1);
        if (save_cap) {
            st_cnt = p.lsaved.as<uint32_t>();
            st_d = (float*)(p.lsaved.as<char>() + ((nq * 4 + 255) & ~(size_t)255));
            st_i = (uint32_t*)(st_d + (size_t)nq * save_cap);
        }
        if (split) {
            CUDA_CHECK(cudaStreamCreateWithFlags(&p.aux, cudaStreamNonBlocking));
            CUDA_CHECK(cudaEventCreateWithFlags(&p.ev_fork, cudaEventDisableTiming));
            CUDA_CHECK(cudaEventCreateWithFlags(&p.ev_join, cudaEventDisableTiming));
        }
        p.budget_levels = levels;
        mlp_layer_tc_prepare();
    }
    // scan scratch sized outside the capture (both scans take nq + 1 entries)
    exclusive_scan_u64(d_total, d_resoff, nq + 1, s, p.tmp);
    exclusive_scan_u32_to_u64(d_rcount, p.d_out_off, nq + 1, s, p.tmp);
    const int dm = L.int8 ? 3 : L.mixed ? 2 : L.fusedsimd ? 1 : 0;
    const void* kfun = phase_a_kernel(L.fast, dm, L.r2);
    CUDA_CHECK(cudaFuncSetAttribute(kfun, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem_a));
    int per_sm = 1;
    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfun, L.wpb * 32, L.smem_a));
    L.grid_a = (uint32_t)std::max<size_t>(1, std::min<size_t>((nq + L.wpb - 1) / L.wpb, (size_t)nsm * std::max(per_sm, 1)));
    KCta kc = ix.wide ? pick_bc<uint64_t>(L.fusedsimd, L.counts, L.mixed) : pick_bc<uint32_t>(L.fusedsimd, L.counts, L.mixed);
    if (stream) {
        p.sb.reserve((uint32_t)nq, v.dim, nq * L.mstride, stream_max_chunks(nq * L.tmax, nq * L.mstride));
        stream_prepare(v, ix.wide, L.fusedsimd);
        // the scan's scratch sized outside the capture
        exclusive_scan_u32_to_u64(p.sb.cnt.as<uint32_t>(), p.sb.coff.as<uint64_t>(), nq * L.mstride + 1, s, p.sb.tmp);
    } else {
        CUDA_CHECK(cudaFuncSetAttribute(kc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem_bc));
        per_sm = 1;
        CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kc, 256, L.smem_bc));
        L.grid_bc = (uint32_t)std::min<size_t>(nq, (size_t)nsm * std::max(per_sm, 1));
    }
    void (*kov)(DevView, const float*, uint32_t, uint32_t, const uint32_t*, const uint32_t*, const uint32_t*,
                const uint64_t*, float, uint32_t, uint32_t, uint32_t*, uint32_t*, uint32_t*, size_t, uint64_t*,
                uint32_t*, uint32_t*, const uint32_t*, SearchCounters*, const uint32_t*, uint32_t*);
    if (ix.wide) kov = L.fusedsimd ? k_phase_bc<uint64_t, true> : k_phase_bc<uint64_t, false>;
    else kov = L.fusedsimd ? k_phase_bc<uint32_t, true> : k_phase_bc<uint32_t, false>;
    CUDA_CHECK(cudaStreamSynchronize(s));

    // ---- record ----
    CUDA_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
    SearchCounters* ctr = p.ctr.as<SearchCounters>();
    CUDA_CHECK(cudaMemsetAsync(ctr, 0, sizeof(SearchCounters), s));
    CUDA_CHECK(cudaMemsetAsync(d_total, 0, (nq + 1) * 8, s));
    CUDA_CHECK(cudaMemsetAsync(d_rcount, 0, (nq + 1) * 4 + 32, s));
    CUDA_CHECK(cudaMemsetAsync(flag, 0, 4, s));
    k_plan_inputs<<<(unsigned)((nq + 255) / 256), 256, 0, s>>>(p.d_m, p.d_ef, (uint32_t)nq, L.mmax, p.ef_max, pm, pef,
                                                               flag);
    // the per-call column of kdist(p, k-1) (hrnn.h:286-293): features and verification
    k_kdist_column<<<(unsigned)((ix.cur + 255) / 256), 256, 0, s>>>(v, L.kidx, p.kcol.as<float>());
    const PhaseA pa{L.fast, dm, L.r2, v, p.d_q, pm, pef, L.efc, L.mstride, p.prox.as<uint32_t>(),
                    p.nprox.as<uint32_t>(), ctr};
    if (!bud) {
        launch_phase_a(pa, L.grid_a, (int)L.wpb, L.vc, L.smem_a, s, (uint32_t)nq, nullptr, 0, 0, 0, nullptr, d_next + 4,
                       0, nullptr, nullptr, nullptr, 0, nullptr);
    } else {
        // frontier pass, features, MLP, decision (search_batch's learned path)
        CUDA_CHECK(cudaMemsetAsync(p.lfb.p, 0, 64, s));
        launch_phase_a(pa, L.grid_a, (int)L.wpb, L.vc, L.smem_a, s, (uint32_t)nq, nullptr,
                       L.two_pass ? bud->m[1] : 0, L.two_pass ? bud->ef : 0, kFrontier, proxd, d_next + 4, save_cap,
                       st_cnt, st_d, st_i, 0, nullptr);
        k_budget_features<<<(unsigned)((nq * 32 + 255) / 256), 256, 0, s>>>(
            v, p.d_q, (uint32_t)nq, p.prox.as<uint32_t>(), proxd, p.nprox.as<uint32_t>(), L.mstride,
            p.kcol.as<float>(), bud->proj.as<float>(), feat);
        float* xn = mlpw;
        float* z1 = xn + nq * kMlpIn;
        float* a1 = z1 + nq * kMlpH;
        float* z2 = a1 + nq * kMlpH;
        float* a2 = z2 + nq * kMlpH;
        float* z3 = a2 + nq * kMlpH;
        bud->mlp.forward_into(feat, (int)nq, xn, z1, a1, z2, a2, z3, s);
        k_budget_decide<<<(unsigned)((nq + 255) / 256), 256, 0, s>>>(z3, (uint32_t)nq, bud->confidence, bud->m[0],
                                                                     bud->m[1], pm, L.two_pass ? 1 : 0,
                                                                     p.nprox.as<uint32_t>(), fb_list, fb_count, levels,
                                                                     grp);
        if (L.two_pass) {
            // the second search over the listed queries; their count is read on the device
            cudaStream_t ls = s;
            if (split) {
                CUDA_CHECK(cudaEventRecord(p.ev_fork, s));
                CUDA_CHECK(cudaStreamWaitEvent(p.aux, p.ev_fork, 0));
                ls = p.aux;
            }
            launch_phase_a(pa, L.grid_a, (int)L.wpb, L.vc, L.smem_a, ls, (uint32_t)nq, fb_list, 0, 0, 0, nullptr,
                           d_next + 5, save_cap, st_cnt, st_d, st_i, save_cap ? 1 : 0, fb_count);
            if (split) CUDA_CHECK(cudaEventRecord(p.ev_join, p.aux));
        }
    }
    uint64_t* resbuf = p.res.as<uint64_t>();
    uint32_t* ovl = flag + 4;  // the overflow list (nq entries) after the clamp flag
    // posting counts, slices and verification of the queries with g[q] == want (all
    // for g null); base: group 0's offsets, which group 1's slices follow
    auto verify_group = [&](const uint8_t* g, uint8_t want, uint64_t* tot, uint64_t* totc, uint64_t* roff,
                            const uint64_t* base) {
        const size_t npairs = nq * L.mstride;
        auto kb = ix.wide ? k_phase_b_count<uint64_t> : k_phase_b_count<uint32_t>;
        kb<<<(unsigned)((npairs + 255) / 256), 256, 0, s>>>(v, (uint32_t)nq, p.d_kp, L.mstride, p.prox.as<uint32_t>(),
                                                            p.nprox.as<uint32_t>(), p.plen.as<uint32_t>(), tot, g,
                                                            want);
        k_cap_totals<<<(unsigned)((nq + 1 + 255) / 256), 256, 0, s>>>(tot, (uint32_t)nq + 1, qcap, totc);
        exclusive_scan_u64(totc, roff, nq + 1, s, p.tmp);
        if (base) k_add_base<<<(unsigned)((nq + 1 + 255) / 256), 256, 0, s>>>(roff, (uint32_t)nq + 1, base);
        if (stream)
            stream_verify(v, ix.wide, L.fusedsimd, p.d_q, (uint32_t)nq, L.mstride, p.prox.as<uint32_t>(),
                          p.plen.as<uint32_t>(), roff, p.kcol.as<float>(), L.kidx, resbuf, d_rcount, ovl,
                          d_next + 1, ctr, p.sb, nsm, s, g, want);
        else
            kc<<<L.grid_bc, 256, L.smem_bc, s>>>(v, p.d_q, (uint32_t)nq, L.mstride, p.prox.as<uint32_t>(),
                                                 p.nprox.as<uint32_t>(), p.plen.as<uint32_t>(), tot, roff,
                                                 p.threshold, p.kcol.as<float>(), L.kidx, resbuf, d_rcount, d_next,
                                                 ovl, d_next + 1, ctr);
        kov<<<(unsigned)(slots / 4), 128, L.smem_w, s>>>(v, p.d_q, 0, L.mstride, p.prox.as<uint32_t>(),
                                                          p.nprox.as<uint32_t>(), p.plen.as<uint32_t>(), roff,
                                                          p.threshold, L.kidx, L.hcap, p.hkey.as<uint32_t>(),
                                                          p.hcnt.as<uint32_t>(), p.lp.as<uint32_t>(), L.tmax, resbuf,
                                                          d_rcount, d_next + 2, ovl, ctr, d_next + 1, flag);
    };
    const uint64_t* pack_off = d_resoff;
    if (split) {
        verify_group(grp, 0, d_total, d_totc, d_resoff, nullptr);
        CUDA_CHECK(cudaStreamWaitEvent(s, p.ev_join, 0));
        CUDA_CHECK(cudaMemsetAsync(d_total2, 0, (nq + 1) * 8, s));
        CUDA_CHECK(cudaMemsetAsync(d_next, 0, 12, s));  // the verification's counters of group 0
        verify_group(grp, 1, d_total2, d_totc2, d_resoff2, d_resoff + nq);
        k_merge_offsets<<<(unsigned)((nq + 255) / 256), 256, 0, s>>>(grp, (uint32_t)nq, d_resoff, d_resoff2,
                                                                     d_resoffm);
        pack_off = d_resoffm;
    } else {
        verify_group(nullptr, 0, d_total, d_totc, d_resoff, nullptr);
    }
    exclusive_scan_u32_to_u64(d_rcount, p.d_out_off, nq + 1, s, p.tmp);
    k_pack_results_capped<<<(unsigned)nq, 128, 0, s>>>((uint32_t)nq, pack_off, d_rcount, p.d_out_off, resbuf,
                                                        p.d_out_lab, p.cap);
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(s, &g);  // leave the stream usable
        if (g) cudaGraphDestroy(g);
        throw;
    }
    const cudaError_t ce = cudaStreamEndCapture(s, &p.graph);
    if (ce != cudaSuccess) fail(HRNN_ERR_CUDA, std::string("search plan: capture failed: ") + cudaGetErrorString(ce));
    CUDA_CHECK(cudaGraphInstantiate(&p.exec, p.graph, 0));
    // kernel nodes of the graph (the launches of one run)
    size_t nn = 0;
    CUDA_CHECK(cudaGraphGetNodes(p.graph, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    if (nn) CUDA_CHECK(cudaGraphGetNodes(p.graph, nodes.data(), &nn));
    p.kernel_nodes = 0;
    for (auto nd : nodes) {
        cudaGraphNodeType t;
        CUDA_CHECK(cudaGraphNodeGetType(nd, &t));
        if (t == cudaGraphNodeTypeKernel) ++p.kernel_nodes;
    }
    p.generation = ix.generation;
}

void plan_run(SearchPlan& p, cudaStream_t s) {
    if (p.generation != p.ix->generation)
        fail(HRNN_ERR_STATE, "search plan: the index changed after the plan was made; make a new plan");
    CUDA_CHECK(cudaGraphLaunch(p.exec, s));
}

uint64_t plan_result(SearchPlan& p, cudaStream_t s, int* clamped) {
    CUDA_CHECK(cudaStreamSynchronize(s));
    uint64_t total = 0;
    uint32_t flag = 0;
    CUDA_CHECK(cudaMemcpy(&total, p.d_out_off + p.nq, 8, cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(&flag, p.inputs.as<uint32_t>() + 2 * p.nq, 4, cudaMemcpyDeviceToHost));
    if (clamped) *clamped = flag ? 1 : 0;
    return total;
}

}  // namespace hrnn
