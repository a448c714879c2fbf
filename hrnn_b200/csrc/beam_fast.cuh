// Two-parent best-first search of level 0 for the reduced-precision search forms
// (INT8 / BF16 rows).  Their proxies only choose candidates -- every returned
// point is decided exactly afterwards -- so this search is free to differ from
// searchBaseLayerST's sequential order (hrnn.h:484-616), which the exact form's
// beam.cuh keeps:
//
//   * each step expands the two best unexpanded beam entries together: both link
//     rows are loaded at once and all their fresh neighbours (up to 64) are
//     scored in one memory round trip (INT8 rows read by eight lanes each), so a step costs
//     one dependent row-gather latency for two expansions;
//   * a scored neighbour enters the beam when it is closer than a full beam's last
//     entry (no per-neighbour sequential acceptance count), duplicates within a
//     step are merged with __match_any_sync, duplicates of beam entries by the
//     equal-distance check;
//   * the beam can be saved after a search with a small beam and resumed later
//     with a larger one (the learned budget's fallback continues the frontier
//     search instead of starting over).
// The search ends when no unexpanded entry is left in the beam, like the
// reference's stop rule (cand_dist > lowerBound with a full result heap).
#pragma once

#include "beam.cuh"

namespace hrnn {

// Per-warp shared memory of the two-parent search:
// q | q8 (dim bytes, padded to 16) | qm | td[efc+32] | ti[efc+32] | vis[vc] | nd[64] | ni[64] | apos[32]
__host__ __device__ inline size_t fast_smem_bytes(uint32_t dim, uint32_t efc, uint32_t vc) {
    return (size_t)dim * 4 + (((size_t)dim + 15) & ~(size_t)15) + 16 + (size_t)(efc + 32) * 8 + (size_t)vc * 4 +
           64 * 8 + 32 * 4;
}

__device__ inline WarpSmem carve_fast(char* base, uint32_t dim, uint32_t efc, uint32_t vc) {
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
    base += 64 * 4;
    s.ni = (uint32_t*)base;
    base += 64 * 4;
    s.apos = (uint32_t*)base;
    return s;
}

// ids[0..cnt) (cnt <= 64) scored with cooperative row reads (coop_i8_load): a
// block of 32 rows in eight load rounds, four whole rows per load instruction.
// R2: both blocks' loads issued before either is scored (one memory round trip
// for 64 rows, twice the registers); otherwise block by block.
template <int NB, bool R2>
__device__ __forceinline__ void warp_i8_coop(const DevView& v, const int* q8, float4 qm, const uint32_t* ids,
                                             uint32_t cnt, float* dout) {
    const int g = (threadIdx.x >> 3) & 3;
    const int4 qw = coop_q_words<NB>(q8);
    const uint32_t r = coop_row();
    const uint32_t nb = cnt > 32 ? 2 : 1;
    auto finish = [&](const int4 (&x)[8], float4 m, uint32_t b0) {
        int p[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) p[i] = dp4a4(x[i], qw);
        const int d = coop_sum8(p);
        if (b0 + r < cnt) dout[b0 + r] = qm.x + m.x * m.x * m.z - 2.f * qm.y * m.x * (float)d;
    };
    if constexpr (R2) {
        int4 x0[8], x1[8];
        float4 m0, m1 = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const uint32_t t = 4 * i + g;
            x0[i] = coop_i8_load<NB>(v.vec_i8, ids[t < cnt ? t : 0]);
        }
        m0 = __ldg(v.i8_meta + ids[r < cnt ? r : 0]);
        if (nb > 1) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const uint32_t t = 32 + 4 * i + g;
                x1[i] = coop_i8_load<NB>(v.vec_i8, ids[t < cnt ? t : 0]);
            }
            m1 = __ldg(v.i8_meta + ids[32 + r < cnt ? 32 + r : 0]);
        }
        finish(x0, m0, 0);
        if (nb > 1) finish(x1, m1, 32);
    } else {
        for (uint32_t b0 = 0; b0 < 32 * nb; b0 += 32) {
            int4 x[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const uint32_t t = b0 + 4 * i + g;
                x[i] = coop_i8_load<NB>(v.vec_i8, ids[t < cnt ? t : 0]);
            }
            const float4 m = __ldg(v.i8_meta + ids[b0 + r < cnt ? b0 + r : 0]);
            finish(x, m, b0);
        }
    }
}

// Scores ids[0..cnt) (cnt <= 64) with the form's rows: DM 3 INT8, DM 2 BF16.
// R2: all 64 INT8 rows in one memory round trip (at twice the registers and so
// fewer resident warps) or 32 at a time; the launch-shape autotuner picks.
template <int DM, bool R2>
__device__ __forceinline__ void warp_dist_list64(const DevView& v, const float* q, const uint32_t* ids,
                                                 uint32_t cnt, float* dout) {
    if constexpr (DM == 3) {
        const int* q8 = i8_q_words(q, v.dim);
        const float4 qm = *i8_q_meta(q, v.dim);
        // rows of 96 and 128 bytes read cooperatively; other widths one row per
        // lane, 32 at a time
        const uint32_t nw = v.dim >> 4;
        if (nw == 6) warp_i8_coop<6, R2>(v, q8, qm, ids, cnt, dout);
        else if (nw == 8) warp_i8_coop<8, R2>(v, q8, qm, ids, cnt, dout);
        else {
            warp_i8_list(v, q8, qm, ids, min(cnt, 32u), dout);
            if (cnt > 32) warp_i8_list(v, q8, qm, ids + 32, cnt - 32, dout + 32);
        }
        __syncwarp();
    } else {
        warp_dist_list<DM>(v, q, ids, min(cnt, 32u), dout);
        if (cnt > 32) warp_dist_list<DM>(v, q, ids + 32, cnt - 32, dout + 32);
    }
}

// Inserts the scored neighbours nd/ni[0..cnt) (cnt <= 32, one per lane) whose
// distance is below a full beam's last entry; the beam stays sorted and is cut to
// EF.  cursor moves back to the first inserted position.
__device__ __forceinline__ void beam_insert_fast(WarpSmem& s, const float* nd, const uint32_t* ni, uint32_t cnt,
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
    uint32_t okb = __ballot_sync(0xFFFFFFFFu, ok);
    if (!okb) return;
    // the same id twice in this batch (two parents sharing a neighbour that the
    // lossy visited cache did not catch): the lowest lane keeps it
    const uint32_t same = __match_any_sync(0xFFFFFFFFu, ok ? id : kInvalid);
    if (ok && (same & lanemask_lt() & okb)) ok = false;
    if (ok) {
        pos = upper_bound(s.td, tsize, d);
        for (int k = (int)pos - 1; k >= 0 && s.td[k] == d; --k)
            if ((s.ti[k] & kIdMask) == id) {
                ok = false;
                break;
            }
    }
    const uint32_t ab = __ballot_sync(0xFFFFFFFFu, ok);
    if (!ab) return;
    const uint32_t na = __popc(ab);
    uint32_t before = 0;
    if (na > 1) {
        for (uint32_t m = ab; m; m &= m - 1) {
            const int i = __ffs(m) - 1;
            const float di = __shfl_sync(0xFFFFFFFFu, d, i);
            if (di < d || (di == d && i < lane)) before++;
        }
    }
    if (ok) s.apos[before] = pos;
    __syncwarp();
    const uint32_t lo = s.apos[0], amax = s.apos[na - 1];
    const uint32_t newsize = min(tsize + na, EF);
    if (tsize > lo) {
        for (int b = (int)lo + (int)(((tsize - lo - 1) / 32) * 32); b >= (int)lo; b -= 32) {
            const uint32_t k = (uint32_t)b + lane;
            float dk = 0.f;
            uint32_t ik = 0, np = 0xFFFFFFFFu;
            if (k < tsize) {
                dk = s.td[k];
                ik = s.ti[k];
                uint32_t sh = na;
                if (k < amax) {
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
    if (ok && npos < newsize) {
        s.td[npos] = d;
        s.ti[npos] = id;
    }
    tsize = newsize;
    cursor = min(cursor, lo);
    __syncwarp();
}

// Two-parent search of level 0 continuing from the beam s.td/s.ti[0..tsize)
// (sorted; ids carry kExpanded).  The visited cache must hold (at least) the
// beam's ids.  The beam keeps the EF nearest scored points; only its first EX
// (<= EF) are expanded, the rest is a reserve a later search with a larger beam
// can resume from (the first EX entries evolve exactly as in a search with
// EF = EX).  Returns the beam size (<= EF).
template <int DM, bool R2>
__device__ uint32_t beam_search_fast(const DevView& v, WarpSmem& s, uint32_t tsize, uint32_t EF, uint32_t EX,
                                     uint32_t vc, unsigned long long& c_dist, unsigned long long& c_exp) {
    const int lane = threadIdx.x & 31;
    uint32_t cursor = 0;
    for (;;) {
        // the (up to) two best unexpanded entries at or after cursor, among the first EX
        uint32_t par0 = kInvalid, par1 = kInvalid;
        const uint32_t lim = min(tsize, EX);
        for (uint32_t b = cursor; b < lim; b += 32) {
            const uint32_t idx = b + lane;
            const bool u = idx < lim && !(s.ti[idx] & kExpanded);
            uint32_t bal = __ballot_sync(0xFFFFFFFFu, u);
            if (!bal) continue;
            if (par0 == kInvalid) {
                par0 = b + __ffs(bal) - 1;
                bal &= bal - 1;
            }
            if (bal) {
                par1 = b + __ffs(bal) - 1;
                break;
            }
        }
        if (par0 == kInvalid) break;
        const uint32_t c0 = s.ti[par0] & kIdMask;
        const uint32_t c1 = par1 != kInvalid ? (s.ti[par1] & kIdMask) : kInvalid;
        cursor = (par1 != kInvalid ? par1 : par0) + 1;
        __syncwarp();
        if (lane == 0) {
            s.ti[par0] |= kExpanded;
            if (par1 != kInvalid) s.ti[par1] |= kExpanded;
        }
        c_exp += par1 != kInvalid ? 2 : 1;
        // both link rows in one go (rows of at most 33 words, maxM0 <= 32)
        uint32_t ra0 = 0, ra1 = 0, rb0 = 0, rb1 = 0;
        load_row(v, c0, 0, ra0, ra1);
        if (c1 != kInvalid) load_row(v, c1, 0, rb0, rb1);
        uint32_t cnt = 0;
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const uint32_t w0 = r ? rb0 : ra0, w1 = r ? rb1 : ra1;
            const uint32_t size = r && c1 == kInvalid ? 0u : (__shfl_sync(0xFFFFFFFFu, w0, 0) & 0xFFFFu);
            const uint32_t a = __shfl_sync(0xFFFFFFFFu, w0, (lane + 1) & 31);
            const uint32_t bw = __shfl_sync(0xFFFFFFFFu, w1, 0);
            const uint32_t nid = (uint32_t)lane < size ? (lane < 31 ? a : bw) : kInvalid;
            const uint32_t slot = hash32(nid) & (vc - 1);
            const bool fresh = (uint32_t)lane < size && s.vis[slot] != nid;
            __syncwarp();
            const uint32_t fb = __ballot_sync(0xFFFFFFFFu, fresh);
            if (fresh) {
                s.ni[cnt + __popc(fb & lanemask_lt())] = nid;
                s.vis[slot] = nid;
            }
            cnt += __popc(fb);
            __syncwarp();
        }
        if (cnt == 0) continue;
        warp_dist_list64<DM, R2>(v, s.q, s.ni, cnt, s.nd);
        c_dist += cnt;
        beam_insert_fast(s, s.nd, s.ni, min(cnt, 32u), EF, tsize, cursor);
        if (cnt > 32) beam_insert_fast(s, s.nd + 32, s.ni + 32, cnt - 32, EF, tsize, cursor);
    }
    return tsize;
}

}  // namespace hrnn
