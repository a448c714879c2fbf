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
//            k_bucket_* group them by target; k_merge_cta (one CTA per target)
//            drops duplicates and ids already listed, selects the K-th distance
//            of list U proposals by radix selection, sorts only the proposals at
//            or below it and merges them into the sorted list keeping K, marking
//            the inserted entries new.  Chunks bound the proposal buffer; lists
//            fill during the first chunk, after which the threshold filters.
//
// Equal distances between different ids are the one place where the bulk merge and
// the sequential insertion can order entries differently (and where the chunk
// boundaries can change which of two equal-distance proposals is kept).
#include <algorithm>
#include <cfloat>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "beam.cuh"
#include "index.hpp"
#include "join.cuh"

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
// thr[nbr]: the farthest entry of nbr's list, FLT_MAX when not full (so an empty
// list never passes `d > thr`).  The decision of every entry is kept in rbits
// (bit j % 32 of word i * ceil(K / 32) + j / 32), so the fill pass reads one word
// per 32 entries instead of their distances and the thresholds of their ids.
__global__ void k_sample_count(const uint32_t* __restrict__ ids, const float* __restrict__ dist,
                               const uint32_t* __restrict__ hdr, const uint8_t* __restrict__ isnew, uint32_t n,
                               uint32_t K, const float* __restrict__ thr, uint32_t* __restrict__ rcount,
                               uint32_t* __restrict__ rbits) {
    size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t wpn = (K + 31) >> 5;
    for (size_t i = warp; i < n; i += nw) {
        uint32_t c = hdr[i] & 0xFFFFu;
        for (uint32_t base = 0; base < c; base += 32) {  // uniform over the warp
            const uint32_t j = base + lane;
            bool rc = false;
            if (j < c) {
                const uint32_t nbr = ids[i * K + j];
                rc = dist[i * K + j] > thr[nbr];
                if (rc) atomicAdd(&rcount[2 * (size_t)nbr + (isnew[i * K + j] ? 0 : 1)], 1u);
            }
            const uint32_t b = __ballot_sync(0xFFFFFFFFu, rc);
            if (lane == 0) rbits[i * wpn + (base >> 5)] = b;
        }
    }
}

// Forward samples (first S new / first S old by rank), reverse-candidate scatter,
// and clearing of the new flags.
__global__ void k_sample_fill(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ rbits,
                              const uint32_t* __restrict__ hdr, uint8_t* __restrict__ isnew, uint32_t n, uint32_t K,
                              uint32_t S, uint32_t cap, uint32_t* __restrict__ newl, uint32_t* __restrict__ newc,
                              uint32_t* __restrict__ oldl, uint32_t* __restrict__ oldc,
                              const uint64_t* __restrict__ roff, uint32_t* __restrict__ rcur,
                              uint32_t* __restrict__ rbuf) {
    size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t wpn = (K + 31) >> 5;
    for (size_t i = warp; i < n; i += nw) {
        uint32_t c = hdr[i] & 0xFFFFu;
        uint32_t nn = 0, no = 0;
        for (uint32_t base = 0; base < c; base += 32) {
            uint32_t j = base + lane;
            bool valid = j < c;
            const uint32_t rb = rbits[i * wpn + (base >> 5)];  // the count pass's decisions
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
            if (valid && ((rb >> lane) & 1u)) {
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
// forward samples (nn_old then stays within 2R = S + R, hrnn.h:1816-1817), one
// warp per node, for R <= kRevSel: the R-th smallest owner by four 8-bit radix
// passes over the segment (owners are distinct within a segment), the owners at or
// below it collected, then placed by rank.  Also sums |new| + |old| over the
// nodes into *entries.
constexpr uint32_t kRevSel = 128;

__global__ void __launch_bounds__(256) k_sample_rev_sel(uint32_t n, uint32_t R, uint32_t cap,
                                                        const uint64_t* __restrict__ roff,
                                                        const uint32_t* __restrict__ rbuf,
                                                        uint32_t* __restrict__ newl, uint32_t* __restrict__ newc,
                                                        uint32_t* __restrict__ oldl, uint32_t* __restrict__ oldc,
                                                        unsigned long long* __restrict__ entries) {
    // entries[0]: |new| + |old| summed over the nodes; entries[2]: the join's
    // pairs |new| (|new| - 1) / 2 + |new| |old| summed (an upper bound: pairs of
    // equal ids are skipped by the join)
    __shared__ uint32_t hist_all[8][256];
    __shared__ uint32_t pick_all[8][kRevSel];
    const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
    uint32_t* hist = hist_all[wl];
    uint32_t* pick = pick_all[wl];
    unsigned long long my_entries = 0, my_pairs = 0;
    const size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t i = warp; i < n; i += nw) {
        uint32_t fin[2] = {0, 0};
        for (int type = 0; type < 2; ++type) {
            const size_t seg = 2 * i + type;
            const uint64_t b = roff[seg];
            const uint32_t len = (uint32_t)(roff[seg + 1] - b);
            uint32_t* L = type == 0 ? newl : oldl;
            uint32_t* C = type == 0 ? newc : oldc;
            const uint32_t base = C[i];
            const uint32_t take = min(len, R);
            if (take > 0) {
                // threshold: the take-th smallest owner (all of them when len <= R)
                uint32_t T = 0xFFFFFFFFu;
                if (len > R) {
                    uint32_t prefix = 0, mask = 0, rank = R;
                    for (int shift = 24; shift >= 0; shift -= 8) {
#pragma unroll
                        for (int k = 0; k < 8; ++k) hist[8 * lane + k] = 0;
                        __syncwarp();
                        for (uint32_t x = lane; x < len; x += 32) {
                            const uint32_t v = rbuf[b + x];
                            if ((v & mask) == prefix) atomicAdd(&hist[(v >> shift) & 255u], 1u);
                        }
                        __syncwarp();
                        uint32_t loc[8], sum = 0;
#pragma unroll
                        for (int k = 0; k < 8; ++k) {
                            loc[k] = hist[8 * lane + k];
                            sum += loc[k];
                        }
                        uint32_t incl = sum;
                        for (int o = 1; o < 32; o <<= 1) {
                            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                            if (lane >= o) incl += y;
                        }
                        const uint32_t excl = incl - sum;
                        uint32_t bin = 0, nrank = 0;
                        const bool mine = excl < rank && rank <= incl;
                        if (mine) {
                            uint32_t r = rank - excl;
#pragma unroll
                            for (int k = 0; k < 8; ++k) {
                                if (r <= loc[k]) {
                                    bin = 8u * lane + (uint32_t)k;
                                    nrank = r;
                                    break;
                                }
                                r -= loc[k];
                            }
                        }
                        const int src = __ffs(__ballot_sync(0xFFFFFFFFu, mine)) - 1;
                        bin = __shfl_sync(0xFFFFFFFFu, bin, src);
                        rank = __shfl_sync(0xFFFFFFFFu, nrank, src);
                        prefix |= bin << shift;
                        mask |= 0xFFu << shift;
                        __syncwarp();
                    }
                    T = prefix;
                }
                // the owners at or below the threshold (exactly `take` of them)
                uint32_t got = 0;
                for (uint32_t x0 = 0; x0 < len; x0 += 32) {
                    const uint32_t x = x0 + lane;
                    const uint32_t v = x < len ? rbuf[b + x] : 0xFFFFFFFFu;
                    const bool keep = x < len && v <= T;
                    const uint32_t bal = __ballot_sync(0xFFFFFFFFu, keep);
                    if (keep) pick[got + __popc(bal & lanemask_lt_())] = v;
                    got += __popc(bal);
                }
                __syncwarp();
                // ascending by rank (distinct values)
                uint32_t v4[kRevSel / 32], r4[kRevSel / 32];
#pragma unroll
                for (int k = 0; k < (int)(kRevSel / 32); ++k) {
                    const uint32_t x = lane + 32u * k;
                    v4[k] = x < take ? pick[x] : 0xFFFFFFFFu;
                    r4[k] = 0;
                }
                for (uint32_t y = 0; y < take; ++y) {
                    const uint32_t w = pick[y];
#pragma unroll
                    for (int k = 0; k < (int)(kRevSel / 32); ++k) r4[k] += w < v4[k] ? 1u : 0u;
                }
#pragma unroll
                for (int k = 0; k < (int)(kRevSel / 32); ++k) {
                    const uint32_t x = lane + 32u * k;
                    if (x < take) L[i * cap + base + r4[k]] = v4[k];
                }
                __syncwarp();
            }
            if (lane == 0) C[i] = base + take;
            my_entries += base + take;
            fin[type] = base + take;
        }
        my_pairs += (unsigned long long)fin[0] * (fin[0] - (fin[0] > 0)) / 2 + (unsigned long long)fin[0] * fin[1];
    }
    if (lane == 0 && my_entries) atomicAdd(entries, my_entries);
    if (lane == 0 && my_pairs) atomicAdd(entries + 2, my_pairs);
}

__global__ void k_sample_rev(uint32_t n, uint32_t R, uint32_t cap, const uint64_t* __restrict__ roff,
                             const uint32_t* __restrict__ rbuf, uint32_t* __restrict__ newl,
                             uint32_t* __restrict__ newc, uint32_t* __restrict__ oldl, uint32_t* __restrict__ oldc,
                             unsigned long long* __restrict__ entries) {
    unsigned long long my_entries = 0, my_pairs = 0;  // as k_sample_rev_sel
    size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t i = warp; i < n; i += nw) {
        uint32_t fin[2] = {0, 0};
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
            my_entries += base + take;
            fin[type] = base + take;
        }
        my_pairs += (unsigned long long)fin[0] * (fin[0] - (fin[0] > 0)) / 2 + (unsigned long long)fin[0] * fin[1];
    }
    if (lane == 0 && my_entries) atomicAdd(entries, my_entries);
    if (lane == 0 && my_pairs) atomicAdd(entries + 2, my_pairs);
}

// ---- phase 2: join -----------------------------------------------------------

// One block (16 warps) per node of the chunk at a time: exact FP32 distances of
// all sample pairs.  The node's rows are staged in shared memory (stride dim + 4
// floats: 16-byte aligned and free of bank conflicts for float4 reads).  Work
// unit: kJR rows i0 .. i0 + 3 (a row tile of the new list) x one column j > i0;
// a tile's columns run from i0 + 1 to the last row, and the units of all tiles
// are numbered consecutively, so a warp takes 32 consecutive units (lane = unit)
// and no lane computes a pair below the diagonal or past the last row.  The row
// vectors are mostly read by the whole warp at one address (broadcast) and the
// lane's column vector once for all kJR pairs, so a 16-byte shared-memory read
// feeds 4 kJR elementwise steps.  Each pair keeps the reference's 16
// accumulators (element e into accumulator e mod 16, then summed left to right),
// so the tiling leaves every distance bit-identical.
//
// NBUF 1 (256 threads, two blocks per SM): one stage per block, the default.
// NBUF 2 (512 threads, one block per SM): two stages, the next node's rows
// copied asynchronously while the current node is computed (a measured option).
// Nodes without new entries have no pairs and are skipped.  Proposals go to
// ranges of the buffer a warp reserves kReserve slots at a time (one atomic per
// range instead of one per tile; a tile's proposals continue in a new range when
// the current one is full); the unused end of a warp's last range is filled with
// target kNoTarget, which the grouping skips.
constexpr int kJR = 4;  // 8 rows (207 registers, one block per SM) measured 1.4x slower
constexpr uint32_t kReserve = 128;
constexpr uint32_t kNoTarget = 0xFFFFFFFFu;

// Units of row tiles 0 .. a-1 (tile t has tot - 1 - kJR t columns).
__device__ __forceinline__ uint32_t join_units_before(uint32_t a, uint32_t tot) {
    return a * (tot - 1) - (kJR / 2) * a * (a - 1);
}

__host__ __device__ inline size_t join_stage_floats(uint32_t dim, uint32_t cap) {
    return (size_t)(2 * cap + kJR) * (dim + 4);
}

__host__ __device__ inline size_t join_smem_bytes(uint32_t dim, uint32_t cap, int nbuf) {
    return (size_t)nbuf * (join_stage_floats(dim, cap) * 4 + (size_t)2 * cap * 8);
}

template <int NBUF>
constexpr int join_threads() {
    return NBUF == 2 ? 512 : 256;
}

template <bool FUSED, int NBUF>
__global__ void __launch_bounds__(join_threads<NBUF>(), NBUF == 2 ? 1 : 2) k_join(const float* __restrict__ vec, uint32_t dim, uint32_t node0,
                                                 uint32_t node1, uint32_t cap, const uint32_t* __restrict__ newl,
                                                 const uint32_t* __restrict__ newc, const uint32_t* __restrict__ oldl,
                                                 const uint32_t* __restrict__ oldc, const float* __restrict__ thr,
                                                 Prop* __restrict__ prop, unsigned long long* __restrict__ pcount,
                                                 unsigned long long pcap, unsigned long long* __restrict__ njoin) {
    extern __shared__ __align__(16) float sm[];
    const uint32_t SP = dim + 4;
    const size_t stage = join_stage_floats(dim, cap);
    // stage b: rows at sm + b stage, then (after all stages) ids and thresholds
    uint32_t* const ids0 = (uint32_t*)(sm + NBUF * stage);
    auto rows_of = [&](int b) { return sm + b * stage; };
    auto ids_of = [&](int b) { return ids0 + (size_t)b * 4 * cap; };
    auto thr_of = [&](int b) { return (float*)(ids0 + (size_t)b * 4 * cap + 2 * cap); };
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t d4 = dim >> 2;
    unsigned long long local_pairs = 0;
    unsigned long long rbase = 0, rend = 0;  // this warp's reserved proposal range (uniform over the warp)

    // ids and thresholds of a node's rows (new first, then old) into stage b
    auto load_ids = [&](uint32_t node, int b, uint32_t nn, uint32_t tot) {
        for (uint32_t r = threadIdx.x; r < tot; r += blockDim.x) {
            const uint32_t id = r < nn ? newl[(size_t)node * cap + r] : oldl[(size_t)node * cap + (r - nn)];
            ids_of(b)[r] = id;
            thr_of(b)[r] = thr[id];
        }
    };
    // the rows themselves, a warp per row and 16 bytes per lane, as asynchronous copies
    auto issue_rows = [&](int b, uint32_t tot) {
        for (uint32_t r = w; r < tot; r += nw) {
            const float4* src = reinterpret_cast<const float4*>(vec + (size_t)ids_of(b)[r] * dim);
            float4* dst = reinterpret_cast<float4*>(rows_of(b) + (size_t)r * SP);
            for (uint32_t c = lane; c < d4; c += 32) {
                const uint32_t sa = (uint32_t)__cvta_generic_to_shared(dst + c);
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(src + c) : "memory");
            }
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    // `cnt` slots for this warp's proposals (warp-uniform call): the rest of the
    // current range first (rem slots from *b1), then a new range from *b2; the
    // proposal at position v of the tile goes to v < rem ? b1 + v : b2 + v - rem,
    // so only the end of the last range is left unused
    auto reserve = [&](uint32_t cnt, unsigned long long& b1, uint32_t& rem, unsigned long long& b2) {
        b1 = rbase;
        rem = (uint32_t)min((unsigned long long)cnt, rend - rbase);
        b2 = 0;
        if (rem < cnt) {
            const uint32_t need = cnt - rem, take = max(need, kReserve);
            unsigned long long t0 = 0;
            if (lane == 0) t0 = atomicAdd(pcount, (unsigned long long)take);
            b2 = __shfl_sync(0xFFFFFFFFu, t0, 0);
            rbase = b2 + need;
            rend = b2 + take;
        } else {
            rbase += cnt;
        }
    };

    auto compute = [&](int b, uint32_t nn, uint32_t tot) {
        const float* R = rows_of(b);
        const uint32_t* ids = ids_of(b);
        const float* th = thr_of(b);
        const uint32_t ntile = (nn + kJR - 1) / kJR;
        const uint32_t F = join_units_before(ntile, tot);
        const uint32_t sp4 = SP >> 2;
        for (uint32_t f0 = 32u * w; f0 < F; f0 += 32u * nw) {
            const uint32_t f = f0 + lane;
            const bool live = f < F;
            // row tile of unit f: the largest a with join_units_before(a) <= f
            uint32_t lo = 0, hi = ntile - 1;
            const uint32_t fc = live ? f : F - 1;
            while (lo < hi) {
                const uint32_t mid = (lo + hi + 1) >> 1;
                if (join_units_before(mid, tot) <= fc) lo = mid;
                else hi = mid - 1;
            }
            const uint32_t i0 = lo * kJR;
            const uint32_t j = i0 + 1 + (fc - join_units_before(lo, tot));
            float acc[kJR][16];
#pragma unroll
            for (int r = 0; r < kJR; ++r)
#pragma unroll
                for (int l = 0; l < 16; ++l) acc[r][l] = 0.f;
            // rows past the staged ones (i0 + r >= tot) read the spare rows at the
            // end of the stage; their sums are never used
            const float4* xb = reinterpret_cast<const float4*>(R + (size_t)j * SP);
            const float4* xa = reinterpret_cast<const float4*>(R + (size_t)i0 * SP);
            for (uint32_t e4 = 0; e4 < d4; e4 += 4) {
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const float4 bb = xb[e4 + c];
#pragma unroll
                    for (int r = 0; r < kJR; ++r) {
                        const float4 aa = xa[(size_t)r * sp4 + e4 + c];
                        acc[r][4 * c + 0] = sq_step(acc[r][4 * c + 0], aa.x - bb.x, FUSED);
                        acc[r][4 * c + 1] = sq_step(acc[r][4 * c + 1], aa.y - bb.y, FUSED);
                        acc[r][4 * c + 2] = sq_step(acc[r][4 * c + 2], aa.z - bb.z, FUSED);
                        acc[r][4 * c + 3] = sq_step(acc[r][4 * c + 3], aa.w - bb.w, FUSED);
                    }
                }
            }
            float dd[kJR];
            uint32_t emit = 0;  // bit 2r: i -> j proposal, bit 2r+1: j -> i
            const uint32_t bj = ids[j];
            const float tj = th[j];
#pragma unroll
            for (int r = 0; r < kJR; ++r) {
                float dv = acc[r][0];
#pragma unroll
                for (int l = 1; l < 16; ++l) dv = __fadd_rn(dv, acc[r][l]);
                dd[r] = dv;
                const uint32_t i = i0 + r;
                if (live && i < nn && j > i && ids[i] != bj) {
                    local_pairs++;
                    if (dv < th[i]) emit |= 1u << (2 * r);
                    if (dv < tj) emit |= 2u << (2 * r);
                }
            }
            // The tile's proposals grouped by target, so the grouping pass meets
            // long runs of one target: row r's proposals (target ids[i0 + r], the
            // same for most lanes) in block r, then each lane's proposals to its
            // column (target bj) together.
            const uint32_t lt = (1u << lane) - 1u;
            uint32_t rowpos[kJR], nrow = 0;
#pragma unroll
            for (int r = 0; r < kJR; ++r) {
                const uint32_t bal = __ballot_sync(0xFFFFFFFFu, (emit >> (2 * r)) & 1u);
                rowpos[r] = nrow + __popc(bal & lt);
                nrow += __popc(bal);
            }
            const uint32_t nc = __popc(emit & 0xAAu);
            uint32_t incl = nc;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                if (lane >= o) incl += y;
            }
            const uint32_t wt = nrow + __shfl_sync(0xFFFFFFFFu, incl, 31);
            if (wt) {
                unsigned long long b1, b2;
                uint32_t rem;
                reserve(wt, b1, rem, b2);
                auto slot = [&](uint32_t x) { return x < rem ? b1 + x : b2 + (x - rem); };
                uint32_t v = nrow + incl - nc;  // this lane's first column-block position
#pragma unroll
                for (int r = 0; r < kJR; ++r) {
                    const uint32_t ai = ids[(i0 + r) < tot ? i0 + r : 0];
                    if ((emit >> (2 * r)) & 1u) {
                        const unsigned long long q = slot(rowpos[r]);
                        if (q < pcap) prop[q] = Prop{ai, bj, dd[r]};
                    }
                    if ((emit >> (2 * r + 1)) & 1u) {
                        const unsigned long long q = slot(v++);
                        if (q < pcap) prop[q] = Prop{bj, ai, dd[r]};
                    }
                }
            }
        }
    };

    uint32_t node = node0 + blockIdx.x;
    if constexpr (NBUF == 2) {
        // this block's next node with new entries at or after x (uniform over the block)
        auto next_active = [&](uint32_t x) {
            while (x < node1 && newc[x] == 0) x += gridDim.x;
            return x;
        };
        // the first node's stage, then per node: the next node's ids, wait for this
        // node's rows, start the next node's rows, compute
        node = next_active(node);
        uint32_t nn = 0, tot = 0;
        if (node < node1) {
            nn = newc[node];
            tot = nn + oldc[node];
            load_ids(node, 0, nn, tot);
        }
        __syncthreads();
        issue_rows(0, tot);
        int b = 0;
        while (node < node1) {
            const uint32_t nxt = next_active(node + gridDim.x);
            uint32_t nn2 = 0, tot2 = 0;
            if (nxt < node1) {
                nn2 = newc[nxt];
                tot2 = nn2 + oldc[nxt];
                load_ids(nxt, b ^ 1, nn2, tot2);
            }
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
            __syncthreads();  // this node's rows and the next node's ids are in place
            issue_rows(b ^ 1, tot2);
            compute(b, nn, tot);
            __syncthreads();  // stage b is free for the node after next
            b ^= 1;
            node = nxt;
            nn = nn2;
            tot = tot2;
        }
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    } else {
        for (; node < node1; node += gridDim.x) {
            const uint32_t nn = newc[node];
            if (nn == 0) continue;  // no pairs (uniform over the block)
            const uint32_t tot = nn + oldc[node];
            __syncthreads();
            load_ids(node, 0, nn, tot);
            __syncthreads();
            issue_rows(0, tot);
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
            __syncthreads();
            compute(0, nn, tot);
        }
    }
    // the unused end of this warp's range
    for (unsigned long long q = rbase + lane; q < rend; q += 32)
        if (q < pcap) prop[q].target = kNoTarget;
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

// The join emits a pair's proposals next to each other, so a warp's 32
// consecutive proposals name few targets: lanes of the same target share one
// atomic (leader adds the group's size, each lane takes its rank in the group).
// Slots with target kNoTarget (the unused ends of the join's reserved ranges) are
// skipped; `nvalid` (optional) counts the others.
__global__ void k_bucket_count(const Prop* __restrict__ prop, unsigned long long np, uint32_t* __restrict__ tcount,
                               unsigned long long* __restrict__ nvalid) {
    const uint32_t lt = lanemask_lt_();
    uint32_t mine = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t t = prop[i].target;
        const uint32_t peers = __match_any_sync(__activemask(), t);
        if ((peers & lt) == 0 && t != kNoTarget) {
            atomicAdd(&tcount[t], (uint32_t)__popc(peers));
            mine += __popc(peers);
        }
    }
    if (nvalid) {
        for (int o = 16; o; o >>= 1) mine += __shfl_xor_sync(0xFFFFFFFFu, mine, o);
        if ((threadIdx.x & 31) == 0 && mine) atomicAdd(nvalid, (unsigned long long)mine);
    }
}

// Each warp takes kFillU consecutive runs of 32 proposals at a time: their loads,
// then their cursor atomics (independent of each other), then their stores, so a
// warp has kFillU atomic round trips in flight instead of one.
constexpr int kFillU = 4;

__global__ void k_bucket_fill(const Prop* __restrict__ prop, unsigned long long np, const uint64_t* __restrict__ toff,
                              uint32_t* __restrict__ tcur, uint64_t* __restrict__ bucket) {
    const uint32_t lt = lanemask_lt_();
    const int lane = threadIdx.x & 31;
    const size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const size_t nwarps = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t b = warp * (32 * kFillU); b < np; b += nwarps * (32 * kFillU)) {  // uniform over the warp
        Prop p[kFillU];
#pragma unroll
        for (int r = 0; r < kFillU; ++r) {
            const size_t i = b + (size_t)r * 32 + lane;
            p[r] = i < np ? prop[i] : Prop{kNoTarget, 0u, 0.f};
        }
        uint32_t peers[kFillU], base[kFillU];
#pragma unroll
        for (int r = 0; r < kFillU; ++r) {
            peers[r] = __match_any_sync(0xFFFFFFFFu, p[r].target);
            base[r] = 0;
            if ((peers[r] & lt) == 0 && p[r].target != kNoTarget)
                base[r] = atomicAdd(&tcur[p[r].target], (uint32_t)__popc(peers[r]));
        }
#pragma unroll
        for (int r = 0; r < kFillU; ++r) {
            base[r] = __shfl_sync(0xFFFFFFFFu, base[r], __ffs(peers[r]) - 1);
            if (p[r].target == kNoTarget) continue;
            const uint64_t pos = toff[p[r].target] + base[r] + (uint32_t)__popc(peers[r] & lt);
            bucket[pos] = ((uint64_t)__float_as_uint(p[r].d) << 32) | p[r].source;  // d >= 0: bit order = value order
        }
    }
}

// ---- phase 2: merge ----------------------------------------------------------

constexpr int kMT = 256;          // merge CTA threads
constexpr uint64_t kOpRemove = 0x80000000ull;  // reverse-list edit: remove (else add) the owner
constexpr uint32_t kMH = 8192;    // source-id hash slots
constexpr uint32_t kMS = 4096;    // survivor keys

// Proposals one window holds: the hash keeps the list and the window's sources
// at a load of at most 0.6.
__host__ __device__ inline uint32_t merge_window(uint32_t K) {
    const uint32_t w = kMH * 3 / 5 > K ? kMH * 3 / 5 - K : 0;
    return w < kMS ? w : kMS;
}

// surv u64[kMS] | hash u32[kMH] | hist u32[256] | ctl u32[16] | two lists of
// (d f32[K], id u32[K]) | two flag arrays u8[K].
__host__ __device__ inline size_t merge_cta_bytes(uint32_t K) {
    size_t b = (size_t)kMS * 8 + (size_t)kMH * 4 + 256 * 4 + 64 + (size_t)K * 16 + (size_t)K * 2;
    return (b + 15) & ~(size_t)15;
}

__device__ __forceinline__ uint32_t hmix(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    return x;
}

// Bits of the rank-th smallest (1-based) of the non-negative floats Ld[0..cnt) and
// hi32(surv[0..S)) (bit order = value order): four 8-bit radix passes.
__device__ uint32_t block_select(const float* Ld, uint32_t cnt, const uint64_t* surv, uint32_t S, uint32_t rank,
                                 uint32_t* hist, uint32_t* ctl) {
    const int tid = threadIdx.x, lane = tid & 31;
    uint32_t prefix = 0, mask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int i = tid; i < 256; i += kMT) hist[i] = 0;
        __syncthreads();
        for (uint32_t j = tid; j < cnt; j += kMT) {
            const uint32_t b = __float_as_uint(Ld[j]);
            if ((b & mask) == prefix) atomicAdd(&hist[(b >> shift) & 255u], 1u);
        }
        for (uint32_t x = tid; x < S; x += kMT) {
            const uint32_t b = (uint32_t)(surv[x] >> 32);
            if ((b & mask) == prefix) atomicAdd(&hist[(b >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (tid < 32) {
            uint32_t loc[8], sum = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                loc[k] = hist[8 * lane + k];
                sum += loc[k];
            }
            uint32_t incl = sum;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                if (lane >= o) incl += y;
            }
            const uint32_t excl = incl - sum;
            if (excl < rank && rank <= incl) {
                uint32_t r = rank - excl;
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    if (r <= loc[k]) {
                        ctl[3] = 8 * lane + k;
                        ctl[4] = r;
                        break;
                    }
                    r -= loc[k];
                }
            }
        }
        __syncthreads();
        prefix |= ctl[3] << shift;
        mask |= 0xFFu << shift;
        rank = ctl[4];
    }
    return prefix;
}

// One CTA per target with proposals (targets handed out by *next_t).  Each window
// of up to merge_window(K) proposals: drop those at or above the current farthest
// entry (full list), those whose source is listed, and repeated sources (a
// repeated pair has the same distance); find the K-th smallest distance tau of
// (list U survivors) by radix selection; sort the survivors at or below tau by
// (d, source) and merge them into the list, list entries first among equal
// distances, keeping K.  Inserted entries are marked new (isnew may be null).
//
// ops (may be null): the list changes as reverse-list edits for the mutable
// reverse lists -- an inserted entry v of u's list is (v << 32 | u), an entry w it
// pushed out (w << 32 | u | kOpRemove); at most ops_cap are written, *nops counts
// them all.
//
// tlist (may be null): merge only the targets tlist[0 .. *tlist_n) (those the
// warp merge left), instead of every target.
__global__ void __launch_bounds__(kMT) k_merge_cta(uint32_t n, uint32_t K, const uint64_t* __restrict__ toff,
                                                   const uint64_t* __restrict__ bucket, uint32_t* __restrict__ hdr,
                                                   uint32_t* __restrict__ ids, float* __restrict__ dist,
                                                   uint8_t* __restrict__ isnew, unsigned long long* __restrict__ nupd,
                                                   uint32_t* __restrict__ next_t, uint64_t* __restrict__ ops,
                                                   unsigned long long* __restrict__ nops,
                                                   unsigned long long ops_cap, const uint32_t* __restrict__ tlist,
                                                   const uint32_t* __restrict__ tlist_n) {
    extern __shared__ __align__(16) char smraw[];
    uint64_t* surv = (uint64_t*)smraw;
    uint32_t* hk = (uint32_t*)(surv + kMS);
    uint32_t* hist = hk + kMH;
    uint32_t* ctl = hist + 256;  // 0 target, 1 survivors, 2 candidates, 3-4 select, 5 first changed
    float* LdA = (float*)(ctl + 16);
    uint32_t* LiA = (uint32_t*)(LdA + K);
    float* LdB = (float*)(LiA + K);
    uint32_t* LiB = (uint32_t*)(LdB + K);
    uint8_t* LfA = (uint8_t*)(LiB + K);
    uint8_t* LfB = LfA + K;
    const int tid = threadIdx.x;
    const uint32_t W = merge_window(K);
    unsigned long long upd = 0;
    const uint32_t nt = tlist ? *tlist_n : n;
    for (;;) {
        __syncthreads();
        if (tid == 0) ctl[0] = atomicAdd(next_t, 1u);
        __syncthreads();
        if (ctl[0] >= nt) break;
        const uint32_t u = tlist ? tlist[ctl[0]] : ctl[0];
        const uint64_t pb = toff[u], pe = toff[u + 1];
        if (pb == pe) continue;
        float* Ld = LdA;
        uint32_t* Li = LiA;
        uint8_t* Lf = LfA;
        float* Ld2 = LdB;
        uint32_t* Li2 = LiB;
        uint8_t* Lf2 = LfB;
        uint32_t cnt = hdr[u] & 0xFFFFu;
        const uint32_t cnt0 = cnt;
        // Lf: bit 0 the entry's new flag, bit 1 "was in the list before this merge"
        for (uint32_t j = tid; j < cnt; j += kMT) {
            Ld[j] = dist[(size_t)u * K + j];
            Li[j] = ids[(size_t)u * K + j];
            Lf[j] = (uint8_t)((isnew ? isnew[(size_t)u * K + j] : 0) | 2);
        }
        if (tid == 0) ctl[5] = cnt;
        for (uint64_t w0 = pb; w0 < pe; w0 += W) {
            const uint32_t P = (pe - w0) < W ? (uint32_t)(pe - w0) : W;
            __syncthreads();  // the previous window's reads of ctl and the hash are done
            for (uint32_t i = tid; i < kMH; i += kMT) hk[i] = kInvalid;
            if (tid == 0) {
                ctl[1] = 0;
                ctl[2] = 0;
            }
            __syncthreads();
            for (uint32_t j = tid; j < cnt; j += kMT) {  // listed ids (distinct)
                const uint32_t id = Li[j];
                uint32_t sl = hmix(id) & (kMH - 1);
                while (atomicCAS(&hk[sl], kInvalid, id) != kInvalid) sl = (sl + 1) & (kMH - 1);
            }
            __syncthreads();
            const float worst = cnt >= K ? Ld[cnt - 1] : FLT_MAX;
            for (uint32_t x = tid; x < P; x += kMT) {
                const uint64_t key = bucket[w0 + x];
                const float d = __uint_as_float((uint32_t)(key >> 32));
                if (!(d < worst)) continue;
                const uint32_t src = (uint32_t)key;
                uint32_t sl = hmix(src) & (kMH - 1);
                for (;;) {
                    const uint32_t old = atomicCAS(&hk[sl], kInvalid, src);
                    if (old == kInvalid) {
                        surv[atomicAdd(&ctl[1], 1u)] = key;
                        break;
                    }
                    if (old == src) break;
                    sl = (sl + 1) & (kMH - 1);
                }
            }
            __syncthreads();
            const uint32_t S = ctl[1];
            if (S == 0) continue;
            // tau: bits of the K-th smallest distance of list U survivors
            const uint32_t tau = cnt + S > K ? block_select(Ld, cnt, surv, S, K, hist, ctl) : 0xFFFFFFFFu;
            // survivors at or below tau, compacted to the front
            uint64_t loc[kMS / kMT];
#pragma unroll
            for (int k = 0; k < (int)(kMS / kMT); ++k) {
                const uint32_t x = tid + k * kMT;
                loc[k] = x < S ? surv[x] : ~0ull;
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < (int)(kMS / kMT); ++k)
                if (loc[k] != ~0ull && (uint32_t)(loc[k] >> 32) <= tau) surv[atomicAdd(&ctl[2], 1u)] = loc[k];
            __syncthreads();
            const uint32_t C = ctl[2];
            uint32_t PP = 2;
            while (PP < C) PP <<= 1;
            for (uint32_t x = C + tid; x < PP; x += kMT) surv[x] = ~0ull;
            __syncthreads();
            for (uint32_t k = 2; k <= PP; k <<= 1)
                for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                    for (uint32_t x = tid; x < PP; x += kMT) {
                        const uint32_t y = x ^ j;
                        if (y > x) {
                            const uint64_t a = surv[x], b = surv[y];
                            if ((a > b) == ((x & k) == 0)) {
                                surv[x] = b;
                                surv[y] = a;
                            }
                        }
                    }
                    __syncthreads();
                }
            // merge (list entries first among equal distances), keep K
            const uint32_t ncnt = min(cnt + C, K);
            for (uint32_t j = tid; j < cnt; j += kMT) {
                const float d = Ld[j];
                const uint64_t bound = (uint64_t)__float_as_uint(d) << 32;  // candidates with distance < d
                uint32_t l2 = 0, h2 = C;
                while (l2 < h2) {
                    const uint32_t mid = (l2 + h2) >> 1;
                    if (surv[mid] < bound) l2 = mid + 1;
                    else h2 = mid;
                }
                const uint32_t pos = j + l2;
                if (pos < ncnt) {
                    Ld2[pos] = d;
                    Li2[pos] = Li[j];
                    Lf2[pos] = Lf[j];
                }
            }
            for (uint32_t x = tid; x < C; x += kMT) {
                const uint64_t key = surv[x];
                const float d = __uint_as_float((uint32_t)(key >> 32));
                uint32_t l2 = 0, h2 = cnt;  // list entries with distance <= d
                while (l2 < h2) {
                    const uint32_t mid = (l2 + h2) >> 1;
                    if (Ld[mid] <= d) l2 = mid + 1;
                    else h2 = mid;
                }
                const uint32_t pos = x + l2;
                if (pos < ncnt) {
                    Ld2[pos] = d;
                    Li2[pos] = (uint32_t)key;
                    Lf2[pos] = 1;
                    atomicMin(&ctl[5], pos);
                    upd++;
                }
            }
            __syncthreads();
            float* t0 = Ld;
            Ld = Ld2;
            Ld2 = t0;
            uint32_t* t1 = Li;
            Li = Li2;
            Li2 = t1;
            uint8_t* t2 = Lf;
            Lf = Lf2;
            Lf2 = t2;
            cnt = ncnt;
        }
        __syncthreads();
        const uint32_t lo = ctl[5];
        if (ops) {
            // entries kept from before form a prefix of the old list (the merge keeps
            // list order); the old entries after it were pushed out
            if (tid == 0) ctl[6] = 0;
            __syncthreads();
            uint32_t kept_l = 0;
            for (uint32_t j = tid; j < cnt; j += kMT) kept_l += (Lf[j] >> 1) & 1u;
            if (kept_l) atomicAdd(&ctl[6], kept_l);
            __syncthreads();
            const uint32_t kept = ctl[6];
            for (uint32_t j = lo + tid; j < cnt; j += kMT)
                if (!(Lf[j] & 2u)) {
                    const unsigned long long o = atomicAdd(nops, 1ull);
                    if (o < ops_cap) ops[o] = ((uint64_t)Li[j] << 32) | u;
                }
            for (uint32_t j = kept + tid; j < cnt0; j += kMT) {
                const unsigned long long o = atomicAdd(nops, 1ull);
                if (o < ops_cap) ops[o] = ((uint64_t)ids[(size_t)u * K + j] << 32) | u | kOpRemove;
            }
            __syncthreads();
        }
        for (uint32_t j = lo + tid; j < cnt; j += kMT) {
            dist[(size_t)u * K + j] = Ld[j];
            ids[(size_t)u * K + j] = Li[j];
            if (isnew) isnew[(size_t)u * K + j] = Lf[j] & 1u;
        }
        if (tid == 0) hdr[u] = (hdr[u] & 0xFFFF0000u) | cnt;
    }
    for (int o = 16; o; o >>= 1) upd += __shfl_xor_sync(0xFFFFFFFFu, upd, o);
    if ((tid & 31) == 0 && upd) atomicAdd(nupd, upd);
}

// One warp per target with proposals (targets handed out by *next_t): the
// CTA merge's result without block-wide steps, for targets whose proposals below
// the farthest entry (after the first filter) number at most kWS -- the common
// case once lists are full.  Survivors (d < farthest entry of a full list) are
// sorted by (d, source) in shared memory (bitonic, warp-synchronous); repeats are
// adjacent, and a listed source is found among the list entries of exactly its
// distance (a pair's distance is a pure function of the pair, so a listed
// source carries the same distance); each survivor goes after the list entries
// of distance <= its own, each list entry after the survivors below it, and the
// first K are kept.  Targets with more survivors are listed in ovl for the CTA
// merge, their lists untouched.
constexpr int kWW = 8;  // warps per block of the warp merge

// Per-warp shared memory of the warp merge holding WS survivors.
__host__ __device__ inline size_t merge_warp_bytes(uint32_t K, uint32_t WS) {
    return (size_t)WS * 8 + (((size_t)K * 9 + 15) & ~(size_t)15);
}

template <uint32_t kWS>  // survivors a warp merge holds
__global__ void __launch_bounds__(kWW * 32) k_merge_warp(uint32_t n, uint32_t K, const uint64_t* __restrict__ toff,
                                                         const uint64_t* __restrict__ bucket,
                                                         uint32_t* __restrict__ hdr, uint32_t* __restrict__ ids,
                                                         float* __restrict__ dist, uint8_t* __restrict__ isnew,
                                                         unsigned long long* __restrict__ nupd,
                                                         uint32_t* __restrict__ next_t, uint32_t* __restrict__ ovl,
                                                         uint32_t* __restrict__ n_ovl) {
    extern __shared__ __align__(16) char smraw[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    char* base = smraw + (size_t)w * merge_warp_bytes(K, kWS);
    uint64_t* sk = (uint64_t*)base;  // survivor keys: d bits << 32 | source
    float* Ld = (float*)(base + (size_t)kWS * 8);
    uint32_t* Li = (uint32_t*)(Ld + K);
    uint8_t* Lf = (uint8_t*)(Li + K);
    const uint32_t lt = lanemask_lt_();
    unsigned long long upd = 0;
    for (;;) {
        uint32_t u = 0;
        if (lane == 0) u = atomicAdd(next_t, 1u);
        u = __shfl_sync(0xFFFFFFFFu, u, 0);
        if (u >= n) break;
        const uint64_t pb = toff[u], pe = toff[u + 1];
        if (pb == pe) continue;
        const uint32_t cnt = hdr[u] & 0xFFFFu;
        const float worst = cnt >= K ? dist[(size_t)u * K + cnt - 1] : FLT_MAX;
        __syncwarp();  // the previous target's reads of sk / Ld are done
        // survivors: proposals below the farthest entry of a full list
        uint32_t S = 0;
        bool over = false;
        for (uint64_t x0 = pb; x0 < pe; x0 += 32) {
            const uint64_t x = x0 + lane;
            uint64_t key = 0;
            bool keep = false;
            if (x < pe) {
                key = bucket[x];
                keep = __uint_as_float((uint32_t)(key >> 32)) < worst;
            }
            const uint32_t bal = __ballot_sync(0xFFFFFFFFu, keep);
            if (S + __popc(bal) > kWS) {
                over = true;
                break;
            }
            if (keep) sk[S + __popc(bal & lt)] = key;
            S += __popc(bal);
        }
        if (over) {
            if (lane == 0) ovl[atomicAdd(n_ovl, 1u)] = u;
            continue;
        }
        if (S == 0) continue;
        // sort the survivors (bitonic over PP >= S slots, padding ~0)
        uint32_t PP = 32;
        while (PP < S) PP <<= 1;
        for (uint32_t i = S + lane; i < PP; i += 32) sk[i] = ~0ull;
        for (uint32_t j = lane; j < cnt; j += 32) {
            Ld[j] = dist[(size_t)u * K + j];
            Li[j] = ids[(size_t)u * K + j];
            Lf[j] = isnew ? isnew[(size_t)u * K + j] : 0;
        }
        __syncwarp();
        for (uint32_t k = 2; k <= PP; k <<= 1)
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t t = lane; t < PP / 2; t += 32) {
                    const uint32_t i = ((t & ~(j - 1)) << 1) | (t & (j - 1)), y = i | j;
                    const uint64_t a = sk[i], b = sk[y];
                    if ((a > b) == ((i & k) == 0)) {
                        sk[i] = b;
                        sk[y] = a;
                    }
                }
                __syncwarp();
            }
        // drop repeats (adjacent after the sort) and listed sources, compacting in
        // place (a write never passes the read position of a later round: the key
        // before a round's first is carried in a register)
        uint32_t C = 0;
        uint64_t carry = ~0ull;
        for (uint32_t i0 = 0; i0 < S; i0 += 32) {
            const uint32_t i = i0 + lane;
            const uint64_t key = i < S ? sk[i] : ~0ull;
            uint64_t prev = __shfl_up_sync(0xFFFFFFFFu, key, 1);
            if (lane == 0) prev = carry;
            carry = __shfl_sync(0xFFFFFFFFu, key, 31);
            bool keep = i < S && key != prev;
            if (keep) {
                const float d = __uint_as_float((uint32_t)(key >> 32));
                uint32_t lo = 0, hi = cnt;  // list entries with distance <= d
                while (lo < hi) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (Ld[mid] <= d) lo = mid + 1;
                    else hi = mid;
                }
                for (int k2 = (int)lo - 1; k2 >= 0 && Ld[k2] == d; --k2)
                    if (Li[k2] == (uint32_t)key) {
                        keep = false;
                        break;
                    }
            }
            const uint32_t bal = __ballot_sync(0xFFFFFFFFu, keep);
            __syncwarp();
            if (keep) sk[C + __popc(bal & lt)] = key;
            C += __popc(bal);
            __syncwarp();
        }
        if (C == 0) continue;
        const uint32_t ncnt = min(cnt + C, K);
        // survivor x goes to x + (list entries with distance <= its own)
        uint32_t first = K;  // the first position that changes
        for (uint32_t x = lane; x < C; x += 32) {
            const uint64_t key = sk[x];
            const float d = __uint_as_float((uint32_t)(key >> 32));
            uint32_t lo = 0, hi = cnt;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (Ld[mid] <= d) lo = mid + 1;
                else hi = mid;
            }
            const uint32_t pos = x + lo;
            first = min(first, pos);
            if (pos < ncnt) {
                dist[(size_t)u * K + pos] = d;
                ids[(size_t)u * K + pos] = (uint32_t)key;
                if (isnew) isnew[(size_t)u * K + pos] = 1;
                upd++;
            }
        }
        for (int o = 16; o; o >>= 1) first = min(first, __shfl_xor_sync(0xFFFFFFFFu, first, o));
        // list entry j (at or after the first change) goes to j + (survivors below it)
        for (uint32_t j = first + lane; j < cnt; j += 32) {
            const float d = Ld[j];
            const uint64_t bound = (uint64_t)__float_as_uint(d) << 32;
            uint32_t lo = 0, hi = C;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (sk[mid] < bound) lo = mid + 1;
                else hi = mid;
            }
            const uint32_t pos = j + lo;
            if (pos < ncnt) {
                dist[(size_t)u * K + pos] = d;
                ids[(size_t)u * K + pos] = Li[j];
                if (isnew) isnew[(size_t)u * K + pos] = Lf[j];
            }
        }
        if (lane == 0) hdr[u] = (hdr[u] & 0xFFFF0000u) | ncnt;
    }
    for (int o = 16; o; o >>= 1) upd += __shfl_xor_sync(0xFFFFFFFFu, upd, o);
    if (lane == 0 && upd) atomicAdd(nupd, upd);
}

// Groups np proposals by target (count, scan, scatter of (d, source) keys) and
// merges each target's group into its list (k_merge_cta).  tcount / toff / tcur
// hold n + 1 entries; `mid` is recorded between the grouping and the merge.
void bucket_and_merge(uint32_t n, uint32_t K, const Prop* prop, unsigned long long np, DevMem& tcount, DevMem& toff,
                      DevMem& tcur, uint64_t* bucket, DevMem& tmp, uint32_t* hdr, uint32_t* ids, float* dist,
                      uint8_t* isnew, unsigned long long* d_nupd, uint32_t* d_nextt, size_t merge_smem,
                      unsigned merge_grid, int nsm, cudaStream_t s, cudaEvent_t mid, uint64_t* ops = nullptr,
                      unsigned long long* nops = nullptr, unsigned long long ops_cap = 0,
                      unsigned long long* nvalid = nullptr) {
    CUDA_CHECK(cudaMemsetAsync(tcount.p, 0, ((size_t)n + 1) * 4, s));
    CUDA_CHECK(cudaMemsetAsync(tcur.p, 0, ((size_t)n + 1) * 4, s));
    const unsigned gb = (unsigned)std::min<unsigned long long>((np + 255) / 256, (unsigned long long)nsm * 32);
    k_bucket_count<<<gb, 256, 0, s>>>(prop, np, tcount.as<uint32_t>(), nvalid);
    CUDA_LAUNCH_CHECK();
    exclusive_scan_u32_to_u64(tcount.as<uint32_t>(), toff.as<uint64_t>(), (size_t)n + 1, s, tmp);
    k_bucket_fill<<<gb, 256, 0, s>>>(prop, np, toff.as<uint64_t>(), tcur.as<uint32_t>(), bucket);
    CUDA_LAUNCH_CHECK();
    if (mid) CUDA_CHECK(cudaEventRecord(mid, s));
    CUDA_CHECK(cudaMemsetAsync(d_nextt, 0, 4, s));
    // Survivors a warp merge holds: 512 (less shared memory per warp, so three
    // blocks per SM instead of two; targets with more survivors go to the CTA
    // merge) measured 15-20 % faster in the heavy iterations of the 1M x 128,
    // K = 500 build than 1024 (HRNN_MERGE_WS = 256 / 1024 selects another, for
    // measurements).
    static const uint32_t ws = [] {
        const char* e = std::getenv("HRNN_MERGE_WS");
        const unsigned long v = e ? std::strtoul(e, nullptr, 10) : 0;
        return (v == 256 || v == 1024) ? (uint32_t)v : 512u;
    }();
    if (!ops && merge_warp_bytes(K, ws) * kWW <= 227 * 1024) {
        // warp merge for every target, then the CTA merge for the targets it left
        // (tcur and tcount are free after the scatter: the left targets and their count)
        const size_t wsm = merge_warp_bytes(K, ws) * kWW;
        auto kmw = ws == 256 ? k_merge_warp<256> : ws == 512 ? k_merge_warp<512> : k_merge_warp<1024>;
        int per_sm = 1;
        CUDA_CHECK(cudaFuncSetAttribute(kmw, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsm));
        CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kmw, kWW * 32, wsm));
        uint32_t* left = tcur.as<uint32_t>();
        uint32_t* n_left = tcount.as<uint32_t>();
        CUDA_CHECK(cudaMemsetAsync(n_left, 0, 4, s));
        kmw<<<(unsigned)(nsm * std::max(per_sm, 1)), kWW * 32, wsm, s>>>(
            n, K, toff.as<uint64_t>(), bucket, hdr, ids, dist, isnew, d_nupd, d_nextt, left, n_left);
        CUDA_LAUNCH_CHECK();
        CUDA_CHECK(cudaMemsetAsync(d_nextt, 0, 4, s));
        k_merge_cta<<<merge_grid, kMT, merge_smem, s>>>(n, K, toff.as<uint64_t>(), bucket, hdr, ids, dist, isnew,
                                                        d_nupd, d_nextt, nullptr, nullptr, 0, left, n_left);
    } else {
        k_merge_cta<<<merge_grid, kMT, merge_smem, s>>>(n, K, toff.as<uint64_t>(), bucket, hdr, ids, dist, isnew,
                                                        d_nupd, d_nextt, ops, nops, ops_cap, nullptr, nullptr);
    }
    CUDA_LAUNCH_CHECK();
}

int smcount(int dev) {
    int v = 148;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v;
}


// ---- insertPointDynamic (hrnn.h:2360-2534), batched ------------------------
//
// The reference inserts one point at a time under per-node locks: HNSW insertion
// with the KNN-graph seed (addPoint), registration of the point in its
// neighbours' reverse lists, a self-query over the reverse lists of its first
// m_update neighbours (all of them for m_update = 0) that skips the point and its
// neighbours, and for every distinct candidate x_i an exact FP32 distance and
// try_update_knng_evict(x_i, x_new, d) (insert when the list is not full or d is
// below its farthest entry, evicting that entry); with `bidirectional` the new
// point's own list becomes the K nearest of (its list U its candidates).
//
// Here a batch of points is inserted at once: add_points (the GPU HNSW builder),
// a reverse-list rebuild (registers the batch in its neighbours' lists and drops
// evicted entries exactly), then k_dyn_self_query emits the list updates of every
// new point as proposals and bucket_and_merge applies them with the K-smallest
// merge of the NNDescent path (the outcome of a sequence of evicting inserts).
// Points of one batch see each other through the reverse lists but not through
// each other's list updates; the reference's parallel insert loop has no fixed
// order either.

constexpr uint32_t kDX = 4096;  // excluded ids (the point and its list; K <= 2048)
constexpr uint32_t kDC = 8192;  // candidate hash slots
constexpr uint32_t kDB = 2048;  // candidates buffered before their distances are taken

__device__ __forceinline__ bool hset_insert(uint32_t* h, uint32_t cap, uint32_t x) {
    uint32_t sl = hmix(x) & (cap - 1);
    for (uint32_t probes = 0; probes < cap; ++probes) {
        const uint32_t old = atomicCAS(&h[sl], kInvalid, x);
        if (old == kInvalid) return true;
        if (old == x) return false;
        sl = (sl + 1) & (cap - 1);
    }
    return false;  // full: treated as present (the callers keep the load below 0.6)
}

__device__ __forceinline__ bool hset_contains(const uint32_t* h, uint32_t cap, uint32_t x) {
    uint32_t sl = hmix(x) & (cap - 1);
    for (uint32_t probes = 0; probes < cap; ++probes) {
        const uint32_t v = h[sl];
        if (v == x) return true;
        if (v == kInvalid) return false;
        sl = (sl + 1) & (cap - 1);
    }
    return false;
}

// Exact FP32 distance of q (shared memory) to row x in the reference's order: two
// lanes per row for the 16-lane order with dim 96/128/256, else one lane per row.
template <bool FUSED>
__device__ __forceinline__ void dyn_dists(const float* __restrict__ vec, uint32_t dim, int lanes, int fused,
                                          const float* q, const uint32_t* ids, uint32_t cnt, float* out) {
    const int lane = threadIdx.x & 31, p = lane & 1;
    if (lanes == 16 && (dim == 128 || dim == 96 || dim == 256)) {
        for (uint32_t r = 0; r < cnt; r += 16) {
            const uint32_t t = r + (lane >> 1);
            const uint32_t id = ids[t < cnt ? t : r];
            const float* x = vec + (size_t)id * dim;
            float d;
            if (dim == 128) d = l2_pair16<FUSED, 8>(q, x, p);
            else if (dim == 96) d = l2_pair16<FUSED, 6>(q, x, p);
            else d = l2_pair16<FUSED, 16>(q, x, p);
            if (p == 0 && t < cnt) out[t] = d;
        }
    } else {
        for (uint32_t t = lane; t < cnt; t += 32) {
            const float* x = vec + (size_t)ids[t] * dim;
            out[t] = (lanes == 16 && dim % 16 == 0) ? l2_row16<FUSED>(q, x, dim / 16)
                                                    : l2_thread(q, x, dim, lanes, fused);
        }
    }
    __syncwarp();
}

// One CTA per new point x in [x0, x0 + nx) (handed out by *next): the self-query
// and its proposals (x_i <- x when the distance is below x_i's farthest entry,
// and x <- x_i under `bidir`).  The candidate hash dedups within a window of
// about 0.6 kDC candidates; a repeat across windows only repeats a proposal,
// which the merge drops.
template <bool FUSED, class E>
__global__ void __launch_bounds__(256) k_dyn_self_query(
    const float* __restrict__ vec, uint32_t dim, int lanes, int fused, uint32_t x0, uint32_t nx,
    const uint32_t* __restrict__ hdr, const uint32_t* __restrict__ ids, uint32_t K,
    const uint64_t* __restrict__ csr_off, const void* __restrict__ csr_ent_v, uint32_t rb, uint32_t m_update, int bidir,
    const float* __restrict__ thr, Prop* __restrict__ prop, unsigned long long* __restrict__ pcount,
    unsigned long long pcap, unsigned long long* __restrict__ ndist, uint32_t* __restrict__ next,
    const uint32_t* __restrict__ mlen) {
    // mlen non-null: the reverse lists are the mutable ones (owner ids from
    // csr_off[y], mlen[y] of them) instead of the flat CSR
    extern __shared__ __align__(16) char smraw[];
    const E* __restrict__ csr_ent = static_cast<const E*>(csr_ent_v);
    float* q = (float*)smraw;
    uint32_t* xh = (uint32_t*)(q + dim);
    uint32_t* ch = xh + kDX;
    uint32_t* buf = ch + kDC;
    float* bd = (float*)(buf + kDB);
    uint32_t* ctl = (uint32_t*)(bd + kDB);  // 0 point, 1 buffered, 2 hashed since clear
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    constexpr int NW = 8;
    unsigned long long c_dist = 0;
    for (;;) {
        __syncthreads();
        if (tid == 0) ctl[0] = atomicAdd(next, 1u);
        __syncthreads();
        if (ctl[0] >= nx) break;
        const uint32_t x = x0 + ctl[0];
        const uint32_t cnt = hdr[x] & 0xFFFFu;
        const uint32_t P = (m_update > 0 && m_update < cnt) ? m_update : cnt;
        const float tx = thr[x];
        for (uint32_t i = tid; i < dim; i += 256) q[i] = vec[(size_t)x * dim + i];
        for (uint32_t i = tid; i < kDX; i += 256) xh[i] = kInvalid;
        for (uint32_t i = tid; i < kDC; i += 256) ch[i] = kInvalid;
        if (tid == 0) {
            ctl[1] = 0;
            ctl[2] = 0;
        }
        __syncthreads();
        if (tid == 0) hset_insert(xh, kDX, x);
        for (uint32_t j = tid; j < cnt; j += 256) hset_insert(xh, kDX, ids[(size_t)x * K + j]);
        __syncthreads();
        // distances and proposals of the buffered candidates, then an empty buffer
        auto flush = [&]() {
            const uint32_t nb = ctl[1];
            for (uint32_t b0 = w * 32; b0 < nb; b0 += NW * 32) {
                const uint32_t c = min(32u, nb - b0);
                dyn_dists<FUSED>(vec, dim, lanes, fused, q, buf + b0, c, bd + b0);
                uint32_t emit = 0, o = 0;
                float d = 0.f;
                if ((uint32_t)lane < c) {
                    o = buf[b0 + lane];
                    d = bd[b0 + lane];
                    if (d < thr[o]) emit |= 1u;
                    if (bidir && d < tx) emit |= 2u;
                }
                c_dist += (lane == 0) ? c : 0;
                const uint32_t ne = __popc(emit);
                uint32_t incl = ne;
                for (int s2 = 1; s2 < 32; s2 <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, s2);
                    if (lane >= s2) incl += y;
                }
                const uint32_t wt = __shfl_sync(0xFFFFFFFFu, incl, 31);
                if (wt) {
                    unsigned long long base = 0;
                    if (lane == 0) base = atomicAdd(pcount, (unsigned long long)wt);
                    base = __shfl_sync(0xFFFFFFFFu, base, 0);
                    unsigned long long pp = base + (incl - ne);
                    if (emit & 1u) {
                        if (pp < pcap) prop[pp] = Prop{o, x, d};
                        pp++;
                    }
                    if ((emit & 2u) && pp < pcap) prop[pp] = Prop{x, o, d};
                }
            }
            __syncthreads();
            if (tid == 0) ctl[1] = 0;
            if (ctl[2] + 256 > kDC * 3 / 5) {  // window full: start a new one
                for (uint32_t i = tid; i < kDC; i += 256) ch[i] = kInvalid;
                __syncthreads();
                if (tid == 0) ctl[2] = 0;
            }
            __syncthreads();
        };
        for (uint32_t pi = 0; pi < P; ++pi) {
            const uint32_t y = ids[(size_t)x * K + pi];
            const uint64_t b = csr_off[y], e = mlen ? b + mlen[y] : csr_off[y + 1];
            for (uint64_t e0 = b; e0 < e; e0 += 256) {
                if (ctl[1] + 256 > kDB || ctl[2] + 256 > kDC * 3 / 5) flush();
                const uint64_t idx = e0 + tid;
                if (idx < e) {
                    const uint32_t o = mlen ? static_cast<const uint32_t*>(csr_ent_v)[idx]
                                            : (uint32_t)(csr_ent[idx] >> rb);
                    if (!hset_contains(xh, kDX, o) && hset_insert(ch, kDC, o)) {
                        buf[atomicAdd(&ctl[1], 1u)] = o;
                        atomicAdd(&ctl[2], 1u);
                    }
                }
                __syncthreads();
            }
        }
        flush();
    }
    for (int s2 = 16; s2; s2 >>= 1) c_dist += __shfl_xor_sync(0xFFFFFFFFu, c_dist, s2);
    if (lane == 0 && c_dist) atomicAdd(ndist, c_dist);
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
    DevMem isnew, newl, newc, oldl, oldc, rcount, roff, rcur, rbuf, rbits, thr, prop, tcount, toff, tcur, bucket, tmp,
        ctr;
    isnew.alloc((size_t)n * K + 16);
    rbuf.alloc((size_t)n * K * 4 + 16);
    rbits.alloc((size_t)n * ((K + 31) / 32) * 4 + 16);
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
    ctr.alloc(128);  // counters (64 bytes), then the tensor-core join's
    // Proposal buffer: every chunk's lists are merged once, at O(K) per touched
    // target, so few large chunks are cheaper than many small ones.  Up to 2048
    // proposals per node, 2^31 in all, and at most 40% of the free memory
    // (20 bytes per proposal: the record and its bucket key).
    size_t free_b = 0, total_b = 0;
    CUDA_CHECK(cudaMemGetInfo(&free_b, &total_b));
    unsigned long long pcap = std::max<unsigned long long>(
        1 << 20, std::min<unsigned long long>({(unsigned long long)n * 2048, 1ull << 31,
                                               (unsigned long long)(free_b * 0.4 / 20)}));
    if (const char* e = std::getenv("HRNN_REFINE_PCAP")) {  // a smaller buffer (tests of the chunk retries)
        const unsigned long long v = std::strtoull(e, nullptr, 10);
        if (v >= 4096) pcap = std::min(pcap, v);
    }
    // Proposals one chunk aims for (HRNN_REFINE_CHUNK_PROPOSALS, default the whole
    // buffer): smaller chunks merge more often, so lists that start short fill
    // sooner and later chunks are filtered by finite thresholds.
    unsigned long long ptarget = pcap;
    if (const char* e = std::getenv("HRNN_REFINE_CHUNK_PROPOSALS")) {
        const unsigned long long v = std::strtoull(e, nullptr, 10);
        if (v >= 4096) ptarget = std::min(pcap, v);
    }
    prop.alloc(pcap * sizeof(Prop));
    bucket.alloc(pcap * 8);
    uint32_t* hdr = ix.knn_hdr.as<uint32_t>();
    uint32_t* ids = ix.knn_ids.as<uint32_t>();
    float* dist = ix.knn_dist.as<float>();
    unsigned long long* d_njoin = ctr.as<unsigned long long>() + 1;
    unsigned long long* d_nupd = ctr.as<unsigned long long>() + 2;
    uint32_t* d_nextt = (uint32_t*)(ctr.as<unsigned long long>() + 3);  // merge work counter
    unsigned long long* d_pcount = ctr.as<unsigned long long>();  // proposal slots of a chunk
    unsigned long long* d_nprop = ctr.as<unsigned long long>() + 5;  // proposals of the iteration
    const bool fast = ix.order.lanes == 16 && ix.dim % 16 == 0;
    // Tensor-core screened join where the dims and sample sizes allow it.
    const bool tcj = fast && ix.join_mode != kJoinExact && join_tc_supported((uint32_t)ix.dim, cap);
    JoinTcCounters* d_jc = reinterpret_cast<JoinTcCounters*>(ctr.as<char>() + 64);
    // The exact join's two forms: two stages (the next node's rows copied during
    // the current node's pairs) for iterations with many pairs per node, where two
    // stages fit in shared memory; one stage otherwise.  Both persistent (every
    // block resident).
    const bool jf = (ix.order.fused & 1) != 0;
    const bool join2_fits = join_smem_bytes((uint32_t)ix.dim, cap, 2) <= 227 * 1024;
    // The one-stage form (two blocks of 8 warps per SM, each on its own node)
    // measured faster than the two-stage form (16 warps on one node) in every
    // iteration of the 1M x 128, K = 500 build (1.40 s against 1.48 s): the other
    // block's node hides the row loads, and 8 warps share a node's work units
    // with less waiting at its barriers.  HRNN_JOIN2_MIN_PAIRS selects the
    // two-stage form from that many pairs per node (for measurements).
    double join2_min_pairs = 1e300;
    if (const char* e = std::getenv("HRNN_JOIN2_MIN_PAIRS")) join2_min_pairs = std::strtod(e, nullptr);
    const size_t join_smem1 = join_smem_bytes((uint32_t)ix.dim, cap, 1);
    const size_t join_smem2 = join_smem_bytes((uint32_t)ix.dim, cap, 2);
    auto kj1 = jf ? k_join<true, 1> : k_join<false, 1>;
    auto kj2 = jf ? k_join<true, 2> : k_join<false, 2>;
    unsigned join_grid1 = (unsigned)nsm, join_grid2 = (unsigned)nsm;
    if (fast) {
        if (join_smem1 > 227 * 1024) fail(HRNN_ERR_ARG, "refineKNNG: sample size too large for dim");
        int per_sm = 1;
        CUDA_CHECK(cudaFuncSetAttribute(kj1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)join_smem1));
        CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kj1, join_threads<1>(), join_smem1));
        join_grid1 = (unsigned)(nsm * std::max(per_sm, 1));
        if (join2_fits) {
            CUDA_CHECK(cudaFuncSetAttribute(kj2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)join_smem2));
            CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kj2, join_threads<2>(), join_smem2));
            join_grid2 = (unsigned)(nsm * std::max(per_sm, 1));
        }
    }
    // Chunk sizing: proposals per join pair of the last accepted chunk (0 until
    // one is known), so a chunk aims at 70 % of the target even when the pairs per
    // node jump between iterations (a chunk over the buffer is computed twice).
    // Fewer, larger chunks are cheaper: every merge pass reads and writes the
    // lists of all targets it touches.
    double prop_per_pair = 0.0;
    uint32_t retry_cap = UINT32_MAX;  // set when a chunk overflowed the buffer, until it is done
    const size_t merge_smem = merge_cta_bytes(K);
    if (merge_smem > 227 * 1024 || merge_window(K) < 256)
        fail(HRNN_ERR_ARG, "refineKNNG: K_knng too large for the merge kernel");
    CUDA_CHECK(cudaFuncSetAttribute(k_merge_cta, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)merge_smem));
    int merge_per_sm = 1;
    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&merge_per_sm, k_merge_cta, kMT, merge_smem));
    const unsigned merge_grid = (unsigned)(nsm * std::max(merge_per_sm, 1));
    const int g1 = nsm * 16;
    uint32_t chunk = std::max<uint32_t>(1, std::min<uint32_t>(n, 16384));
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
        CUDA_CHECK(cudaMemsetAsync(ctr.p, 0, 128, s));
        // ---- phase 1 ----
        CUDA_CHECK(cudaMemsetAsync(rcount.p, 0, rcount.bytes, s));
        CUDA_CHECK(cudaMemsetAsync(rcur.p, 0, rcur.bytes, s));
        k_thresholds<<<(n + 255) / 256, 256, 0, s>>>(hdr, dist, n, K, thr.as<float>());
        CUDA_LAUNCH_CHECK();
        k_sample_count<<<g1, 256, 0, s>>>(ids, dist, hdr, isnew.as<uint8_t>(), n, K, thr.as<float>(),
                                           rcount.as<uint32_t>(), rbits.as<uint32_t>());
        CUDA_LAUNCH_CHECK();
        exclusive_scan_u32_to_u64(rcount.as<uint32_t>(), roff.as<uint64_t>(), (size_t)2 * n + 1, s, tmp);
        uint64_t rtot = 0;
        CUDA_CHECK(cudaMemcpyAsync(&rtot, roff.as<uint64_t>() + (size_t)2 * n, 8, cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaStreamSynchronize(s));
        rbuf.ensure(std::max<uint64_t>(rtot, 1) * 4);  // rtot <= n K: allocated once up front
        k_sample_fill<<<g1, 256, 0, s>>>(ids, rbits.as<uint32_t>(), hdr, isnew.as<uint8_t>(), n, K, S, cap,
                                          newl.as<uint32_t>(),
                                          newc.as<uint32_t>(), oldl.as<uint32_t>(), oldc.as<uint32_t>(),
                                          roff.as<uint64_t>(), rcur.as<uint32_t>(), rbuf.as<uint32_t>());
        CUDA_LAUNCH_CHECK();
        if (R <= kRevSel)
            k_sample_rev_sel<<<g1, 256, 0, s>>>(n, R, cap, roff.as<uint64_t>(), rbuf.as<uint32_t>(),
                                                 newl.as<uint32_t>(), newc.as<uint32_t>(), oldl.as<uint32_t>(),
                                                 oldc.as<uint32_t>(), ctr.as<unsigned long long>() + 4);
        else
            k_sample_rev<<<g1, 256, 0, s>>>(n, R, cap, roff.as<uint64_t>(), rbuf.as<uint32_t>(), newl.as<uint32_t>(),
                                             newc.as<uint32_t>(), oldl.as<uint32_t>(), oldc.as<uint32_t>(),
                                             ctr.as<unsigned long long>() + 4);
        CUDA_LAUNCH_CHECK();
        CUDA_CHECK(cudaEventRecord(ev[2], s));
        // |new| + |old| summed over nodes (gather bytes of the join) and the join's pairs
        unsigned long long sc[3] = {0, 0, 0};
        CUDA_CHECK(cudaMemcpyAsync(sc, ctr.as<unsigned long long>() + 4, 24, cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaStreamSynchronize(s));
        const unsigned long long sample_entries = sc[0];
        const double pairs_per_node = (double)sc[2] / (double)n;
        t_sample = elapsed(e0, ev[2]);
        unsigned long long njoin_ok = 0;  // pair count after the last accepted chunk
        unsigned long long nprop_ok = 0;  // proposal count after the last accepted chunk
        JoinTcCounters jc_ok{};           // screen counts after the last accepted chunk
        const bool join2 = join2_fits && pairs_per_node >= join2_min_pairs;
        // ---- phase 2, chunk by chunk ----
        for (uint32_t node0 = 0; node0 < n;) {
            if (prop_per_pair > 0.0 && pairs_per_node > 0.0)
                chunk = (uint32_t)std::max(1.0, std::min((double)n, 0.7 * (double)ptarget /
                                                                       (prop_per_pair * pairs_per_node)));
            chunk = std::min(chunk, retry_cap);  // a chunk that overflowed is redone at most this large
            uint32_t node1 = std::min<uint32_t>(n, node0 + chunk);
            k_thresholds<<<(n + 255) / 256, 256, 0, s>>>(hdr, dist, n, K, thr.as<float>());
            CUDA_LAUNCH_CHECK();
            CUDA_CHECK(cudaMemsetAsync(d_pcount, 0, 8, s));
            CUDA_CHECK(cudaEventRecord(ev[3], s));
            unsigned grid = std::min<unsigned>(node1 - node0, (unsigned)nsm * 8);
            if (tcj) {
                join_tc(ix.vec.as<float>(), (uint32_t)ix.dim, node0, node1, cap, newl.as<uint32_t>(),
                        newc.as<uint32_t>(), oldl.as<uint32_t>(), oldc.as<uint32_t>(), thr.as<float>(),
                        prop.as<Prop>(), d_pcount, pcap, d_njoin, d_jc, (ix.order.fused & 1) != 0, ix.join_mode, nsm,
                        s);
            } else if (fast) {
                if (join2)
                    kj2<<<std::min<unsigned>(node1 - node0, join_grid2), join_threads<2>(), join_smem2, s>>>(
                        ix.vec.as<float>(), (uint32_t)ix.dim, node0, node1, cap, newl.as<uint32_t>(),
                        newc.as<uint32_t>(), oldl.as<uint32_t>(), oldc.as<uint32_t>(), thr.as<float>(),
                        prop.as<Prop>(), d_pcount, pcap, d_njoin);
                else
                    kj1<<<std::min<unsigned>(node1 - node0, join_grid1), join_threads<1>(), join_smem1, s>>>(
                        ix.vec.as<float>(), (uint32_t)ix.dim, node0, node1, cap, newl.as<uint32_t>(),
                        newc.as<uint32_t>(), oldl.as<uint32_t>(), oldc.as<uint32_t>(), thr.as<float>(),
                        prop.as<Prop>(), d_pcount, pcap, d_njoin);
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
                // Redo this chunk smaller (the join is pure): np counts every proposal
                // the attempt reserved, so half the buffer at the attempt's own density
                // bounds the retry (the rate that sized the chunk is an average and
                // would size it the same again).
                retry_cap = (uint32_t)std::max(1.0, std::min((double)chunk / 4.0,
                                                             (double)chunk * 0.5 * (double)pcap / (double)np));
                chunk = retry_cap;
                // the pair and screen counts of the dropped attempt start over
                CUDA_CHECK(cudaMemcpyAsync(d_njoin, &njoin_ok, 8, cudaMemcpyHostToDevice, s));
                if (tcj) CUDA_CHECK(cudaMemcpyAsync(d_jc, &jc_ok, sizeof(jc_ok), cudaMemcpyHostToDevice, s));
                CUDA_CHECK(cudaStreamSynchronize(s));
                continue;
            }
            retry_cap = UINT32_MAX;
            const unsigned long long njoin_prev = njoin_ok, nprop_prev = nprop_ok;
            CUDA_CHECK(cudaMemcpyAsync(&njoin_ok, d_njoin, 8, cudaMemcpyDeviceToHost, s));
            if (tcj) CUDA_CHECK(cudaMemcpyAsync(&jc_ok, d_jc, sizeof(jc_ok), cudaMemcpyDeviceToHost, s));
            if (np) {
                bucket_and_merge(n, K, prop.as<Prop>(), np, tcount, toff, tcur, bucket.as<uint64_t>(), tmp, hdr, ids,
                                 dist, isnew.as<uint8_t>(), d_nupd, d_nextt, merge_smem, merge_grid, nsm, s, ev[6],
                                 nullptr, nullptr, 0, d_nprop);
                CUDA_CHECK(cudaEventRecord(ev[5], s));
                CUDA_CHECK(cudaEventSynchronize(ev[5]));
                t_bucket += elapsed(ev[4], ev[6]);
                t_merge += elapsed(ev[6], ev[5]);
            }
            node0 = node1;
            CUDA_CHECK(cudaMemcpyAsync(&nprop_ok, d_nprop, 8, cudaMemcpyDeviceToHost, s));
            CUDA_CHECK(cudaStreamSynchronize(s));
            const unsigned long long chunk_props = nprop_ok - nprop_prev, chunk_pairs = njoin_ok - njoin_prev;
            if (chunk_props && chunk_pairs) {
                prop_per_pair = (double)chunk_props / (double)chunk_pairs;
            } else if (prop_per_pair == 0.0) {
                // no rate yet: keep the chunk's proposals between a quarter and three
                // quarters of the target
                if (chunk_props < ptarget / 4 && chunk < n) chunk = std::min<uint32_t>(n, chunk * 2);
                else if (chunk_props > ptarget / 4 * 3 && chunk > 1) chunk /= 2;
            }
        }
        unsigned long long hc[6] = {0, 0, 0, 0, 0, 0};
        JoinTcCounters hj{};
        CUDA_CHECK(cudaEventRecord(e1, s));
        CUDA_CHECK(cudaMemcpyAsync(hc, ctr.p, 48, cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaMemcpyAsync(&hj, d_jc, sizeof(hj), cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaStreamSynchronize(s));
        if (hj.err) fail(HRNN_ERR_TIMEOUT, "refineKNNG: tensor-core join: wait on the MMA commit expired");
        const double ms = elapsed(e0, e1);
        std::printf("      iter %d: %llu updates, %llu dists  (%.1f ms: sample %.1f, join %.1f, bucket %.1f, "
                    "merge %.1f)\n", it, hc[2], hc[1], ms, t_sample, t_join, t_bucket, t_merge);
        std::fflush(stdout);
        if (it < HRNN_MAX_ITERS) {
            auto& rs = ix.refine_stats;
            rs.iters = it + 1;
            rs.join_dists[it] = hc[1];
            rs.updates[it] = hc[2];
            rs.proposals[it] = hc[5];
            rs.sample_entries[it] = sample_entries;
            rs.ms[it] = ms;
            rs.sample_ms[it] = t_sample;
            rs.join_ms[it] = t_join;
            rs.bucket_ms[it] = t_bucket;
            rs.merge_ms[it] = t_merge;
            rs.screen_survivors[it] = tcj ? hj.survivors : 0;
            rs.screen_dense_nodes[it] = tcj ? hj.dense_nodes : 0;
            rs.screen_misses[it] = tcj ? hj.misses : 0;
            rs.join_mode = tcj ? ix.join_mode : kJoinExact;
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    ix.knng_built = true;                                 // hrnn.h:1861
}

void build_rknng_mutable(Index& ix) {
    if (!ix.knng_built) fail(HRNN_ERR_STATE, "buildRKNNG_mutable: KNNG not built yet");  // hrnn.h:1943-1944
    ix.mr.slack_shift = 0;
    mutable_build(ix);
    ix.rknng_mutable = true;
    uint64_t total = 0;
    if (ix.cur) {
        std::vector<uint32_t> ln(ix.cur);
        CUDA_CHECK(cudaMemcpy(ln.data(), ix.mr.len.p, ix.cur * 4, cudaMemcpyDeviceToHost));
        for (uint32_t x : ln) total += x;
    }
    std::printf("    buildRKNNG_mutable: n=%zu total_entries=%llu\n", ix.cur, (unsigned long long)total);
    std::fflush(stdout);
}

void ensure_flat_rknng(Index& ix) {
    if (ix.csr_stale) {
        build_rknng(ix);
        ix.csr_stale = false;
    }
}

void insert_dynamic(Index& ix, const float* data, const uint64_t* labels, size_t n, unsigned m_update,
                    bool bidirectional) {
    if (!ix.knng_built) fail(HRNN_ERR_STATE, "insertPointDynamic: KNNG not built yet");
    if (!ix.rknng_mutable) fail(HRNN_ERR_STATE, "insertPointDynamic: buildRKNNG_mutable not called");
    if (ix.serve_mode) fail(HRNN_ERR_STATE, "addPoint: index is in serve mode");
    const uint32_t K = (uint32_t)ix.K;
    if (K == 0 || K > kMaxK) fail(HRNN_ERR_ARG, "insertPointDynamic: K_knng must be in [1, 2048]");
    if (ix.cur + n > ix.max_elements)
        fail(HRNN_ERR_LIMIT, "The number of elements exceeds the specified limit");  // hrnn.h:1402-1404
    hrnn_dynamic_stats st{};
    ix.dyn_stats = st;
    if (n == 0) return;
    cudaStream_t s = ix.stream;
    const int nsm = smcount(ix.device);
    const size_t capn = ix.max_elements;
    DevMem thr, prop, bucket, tcount, toff, tcur, tmp, ctr;
    thr.alloc(capn * 4);
    tcount.alloc((capn + 1) * 4);
    toff.alloc((capn + 1) * 8);
    tcur.alloc((capn + 1) * 4);
    ctr.alloc(64);
    size_t free_b = 0, total_b = 0;
    CUDA_CHECK(cudaMemGetInfo(&free_b, &total_b));
    const unsigned long long pcap = std::max<unsigned long long>(
        1 << 20, std::min<unsigned long long>({(unsigned long long)n * 4096, 1ull << 30,
                                               (unsigned long long)(free_b * 0.3 / 20)}));
    prop.alloc(pcap * sizeof(Prop));
    bucket.alloc(pcap * 8);
    if (!ix.mr.valid) mutable_build(ix);
    mutable_ops_reserve(ix, std::min<unsigned long long>(2 * pcap, 1ull << 26));
    unsigned long long* d_pcount = ctr.as<unsigned long long>();
    unsigned long long* d_ndist = d_pcount + 1;
    unsigned long long* d_nupd = d_pcount + 2;
    uint32_t* d_nextt = (uint32_t*)(d_pcount + 3);
    uint32_t* d_next = (uint32_t*)(d_pcount + 4);
    CUDA_CHECK(cudaMemsetAsync(ctr.p, 0, 64, s));
    const size_t merge_smem = merge_cta_bytes(K);
    CUDA_CHECK(cudaFuncSetAttribute(k_merge_cta, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)merge_smem));
    int merge_per_sm = 1;
    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&merge_per_sm, k_merge_cta, kMT, merge_smem));
    const unsigned merge_grid = (unsigned)(nsm * std::max(merge_per_sm, 1));
    const size_t sq_smem = (size_t)ix.dim * 4 + (size_t)(kDX + kDC + 2 * kDB) * 4 + 64;
    const bool fusedsimd = (ix.order.fused & 1) != 0;
    cudaEvent_t ev[4];
    for (auto& e : ev) CUDA_CHECK(cudaEventCreate(&e));
    auto elapsed = [](cudaEvent_t a, cudaEvent_t b) {
        float t = 0.f;
        cudaEventElapsedTime(&t, a, b);
        return (double)t;
    };
    uint32_t chunk = 1024;
    size_t done = 0;
    while (done < n) {
        // Batches of an eighth of the index (at least 4096 points), so that later
        // batches see the earlier ones' updates.
        const size_t sb = std::min(n - done, std::max<size_t>(4096, ix.cur / 8));
        const uint32_t x0 = (uint32_t)ix.cur;
        CUDA_CHECK(cudaEventRecord(ev[0], s));
        add_points(ix, data + done * ix.dim, labels ? labels + done : nullptr, sb);
        CUDA_CHECK(cudaEventRecord(ev[1], s));
        mutable_register(ix, x0, (uint32_t)sb);  // the batch joins its neighbours' reverse lists
        CUDA_CHECK(cudaEventRecord(ev[2], s));
        const uint32_t nall = (uint32_t)ix.cur;
        auto kq = ix.wide ? (fusedsimd ? k_dyn_self_query<true, uint64_t> : k_dyn_self_query<false, uint64_t>)
                          : (fusedsimd ? k_dyn_self_query<true, uint32_t> : k_dyn_self_query<false, uint32_t>);
        CUDA_CHECK(cudaFuncSetAttribute(kq, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sq_smem));
        int sq_per_sm = 1;
        CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sq_per_sm, kq, 256, sq_smem));
        for (uint32_t a = 0; a < sb;) {
            const uint32_t na = (uint32_t)std::min<size_t>(chunk, sb - a);
            k_thresholds<<<(nall + 255) / 256, 256, 0, s>>>(ix.knn_hdr.as<uint32_t>(), ix.knn_dist.as<float>(), nall, K,
                                                           thr.as<float>());
            CUDA_LAUNCH_CHECK();
            CUDA_CHECK(cudaMemsetAsync(d_pcount, 0, 8, s));
            CUDA_CHECK(cudaMemsetAsync(d_next, 0, 4, s));
            const unsigned grid = (unsigned)std::min<size_t>(na, (size_t)nsm * std::max(sq_per_sm, 1));
            kq<<<grid, 256, sq_smem, s>>>(ix.vec.as<float>(), (uint32_t)ix.dim, ix.order.lanes, ix.order.fused,
                                          x0 + a, na, ix.knn_hdr.as<uint32_t>(), ix.knn_ids.as<uint32_t>(), K,
                                          ix.mr.off.as<uint64_t>(), ix.mr.ent.p, 0, m_update,
                                          bidirectional ? 1 : 0, thr.as<float>(), prop.as<Prop>(), d_pcount, pcap,
                                          d_ndist, d_next, ix.mr.len.as<uint32_t>());
            CUDA_LAUNCH_CHECK();
            unsigned long long np = 0;
            CUDA_CHECK(cudaMemcpyAsync(&np, d_pcount, 8, cudaMemcpyDeviceToHost, s));
            CUDA_CHECK(cudaStreamSynchronize(s));
            if (np > pcap) {  // the self-query is pure: redo this chunk smaller
                if (chunk == 1) fail(HRNN_ERR_NOMEM, "insertPointDynamic: proposal buffer too small for one point");
                chunk = std::max<uint32_t>(1, chunk / 4);
                continue;
            }
            if (np) {
                // the merge's list changes are edited into the mutable reverse lists
                bucket_and_merge(nall, K, prop.as<Prop>(), np, tcount, toff, tcur, bucket.as<uint64_t>(), tmp,
                                 ix.knn_hdr.as<uint32_t>(), ix.knn_ids.as<uint32_t>(), ix.knn_dist.as<float>(), nullptr,
                                 d_nupd, d_nextt, merge_smem, merge_grid, nsm, s, nullptr, ix.mr.ops.as<uint64_t>(),
                                 ix.mr.ctl.as<unsigned long long>(), ix.mr.ops_cap);
                mutable_apply(ix);
            }
            st.n_proposals += np;
            a += na;
            if (np < pcap / 4) chunk = std::min<uint32_t>(chunk * 2, 1u << 20);
            else if (np > pcap / 4 * 3 && chunk > 1) chunk /= 2;
        }
        CUDA_CHECK(cudaEventRecord(ev[3], s));
        CUDA_CHECK(cudaEventSynchronize(ev[3]));
        st.insert_ms += elapsed(ev[0], ev[1]);
        st.rknng_ms += elapsed(ev[1], ev[2]);
        st.maintain_ms += elapsed(ev[2], ev[3]);
        st.n_batches++;
        done += sb;
    }
    // The flat CSR the search reads (sorted by rank) is rebuilt once, before its
    // next use (the reference's driver calls buildRKNNG after its inserts,
    // src/hrnn_dynamic_test.cpp:368).
    ix.csr_stale = true;
    ix.rknng_built = true;
    unsigned long long hc[3] = {0, 0, 0};
    CUDA_CHECK(cudaMemcpyAsync(hc, ctr.p, 24, cudaMemcpyDeviceToHost, s));
    CUDA_CHECK(cudaStreamSynchronize(s));
    for (auto& e : ev) cudaEventDestroy(e);
    st.n_inserted = n;
    st.n_dist = hc[1];
    st.n_updates = hc[2];
    ix.rknng_mutable = true;
    ix.dyn_stats = st;
}

}  // namespace hrnn
